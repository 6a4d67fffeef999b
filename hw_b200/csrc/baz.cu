// BAZ pulse encoding for sm_100a.
//
// Restates the field machinery of bazio/encoding (ObjectToBaz.h:60-150 group
// encoder, :373-393 grouping; FieldTransforms.h NoOp / DeltaCompression /
// FloatFixedCodec; FieldSerializers.h TruncateOverflow / SimpleOverflow /
// CompactOverflow) with a runtime field list, the field values of the
// basecaller's Pulse (basecaller/dataTypes/PulseFieldAccessors.h:43-68) and
// the per-ZMW append of PrelimHQFilter / PacketBuffer::AddZmw
// (basecaller/appModules/PrelimHQFilter.cpp:95-118, bazio/writing/PacketBuffer.h:143-210).
//
// One launch, pulse-parallel.  A CTA takes a tile of 128 ZMWs (tiles handed
// out in launch order by a ticket); each of its 256 threads takes a
// contiguous run of the tile's pulses.  A pulse's bytes depend only on the
// pulse and, for delta-coded fields, on the previous kept pulse of its ZMW
// (or the ZMW's state from the previous chunk), so a run is sized on its
// own.  Sweep 1 sizes the runs (pulses loaded four at a time); one block
// scan places the runs in the tile; a decoupled look-back over the tiles
// before it places the tile in the output; sweep 2 writes every run at its
// place (the pulses come from L1/L2 the second time).  The delta state is
// double-buffered: a call reads one copy and writes the other, and the call's
// last tile switches copies when the whole chunk fit in the buffer.
#include <atomic>
#include <string>

#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "hw_device.cuh"

using namespace hwk;

namespace {

constexpr int kMaxFields = 16;
constexpr int kTileRows = 128;       // ZMWs a tile
constexpr int kThreads = 256;        // runs of pulses a tile
constexpr uint64_t kFfNan = 0, kFfInf = 1, kFfNinf = 2, kFfOffset = 3;   // FloatFixedCodec codes
// look-back flags (top two bits of a tile's word): count published, inclusive total published
// kFlagFail: an inclusive word whose prefix is not valid (the tile, or a tile
// before it, gave up waiting); successors stop at it and carry it forward.
constexpr unsigned long long kFlagAgg = 1ull << 62, kFlagInc = 2ull << 62, kFlagFail = 3ull << 62;
constexpr uint32_t kSpinLimit = 1u << 22;  // default bound on polls of a predecessor's status (about 0.4 s)

struct BazSpec
{
    hw_baz_field f[kMaxFields];
    int groupEnd[kMaxFields];     // 1: the field closes its group
    int groupBytes[kMaxFields];   // nominal bytes of the group a field opens (0 elsewhere)
    int slot[kMaxFields];         // delta-state slot of a delta-coded field
    int n;
    int skipRejects;
    int slots;                    // delta-coded fields
};

// ---- field lists: the runtime one, and the basecaller's two as constants ----

struct RtFields
{
    const BazSpec& S;
    __device__ explicit RtFields(const BazSpec& s) : S(s) {}
    __device__ int n() const { return S.n; }
    __device__ hw_baz_field f(int i) const { return S.f[i]; }
    __device__ int groupBytes(int i) const { return S.groupBytes[i]; }
    __device__ bool groupEnd(int i) const { return S.groupEnd[i] != 0; }
    __device__ int slot(int i) const { return S.slot[i]; }
    __device__ bool skip() const { return S.skipRejects != 0; }
    __device__ bool hasDelta() const { return S.slots > 0; }
};

// PulseGroups.h:42-53
struct ProductionFields
{
    __device__ explicit ProductionFields(const BazSpec&) {}
    __host__ __device__ static constexpr int n() { return 3; }
    __host__ __device__ static constexpr hw_baz_field f(int i)
    {
        return i == 0 ? hw_baz_field{HW_BAZ_LABEL, 0, HW_BAZ_NOOP, 0, 0, HW_BAZ_TRUNCATE, 2, 0}
             : i == 1 ? hw_baz_field{HW_BAZ_PULSE_WIDTH, 0, HW_BAZ_NOOP, 0, 0, HW_BAZ_COMPACT_OVERFLOW, 7, 0}
                      : hw_baz_field{HW_BAZ_START_FRAME, 0, HW_BAZ_DELTA, 0, 0, HW_BAZ_COMPACT_OVERFLOW, 7, 0};
    }
    __host__ __device__ static constexpr int groupBytes(int i) { return i == 0 ? 2 : 0; }
    __host__ __device__ static constexpr bool groupEnd(int i) { return i == 2; }
    __host__ __device__ static constexpr int slot(int) { return 0; }
    __host__ __device__ static constexpr bool skip() { return true; }
    __host__ __device__ static constexpr bool hasDelta() { return true; }
};

// PulseGroups.h:55-94
struct InternalFields
{
    __device__ explicit InternalFields(const BazSpec&) {}
    __host__ __device__ static constexpr int n() { return 8; }
    __host__ __device__ static constexpr hw_baz_field f(int i)
    {
        return i < 3 ? ProductionFields::f(i)
             : i == 3 ? hw_baz_field{HW_BAZ_PKMAX, 1, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 8, 2}
             : i == 4 ? hw_baz_field{HW_BAZ_PKMID, 1, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 8, 2}
             : i == 5 ? hw_baz_field{HW_BAZ_PKMEAN, 1, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 8, 2}
             : i == 6 ? hw_baz_field{HW_BAZ_PKVAR, 0, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 7, 2}
                      : hw_baz_field{HW_BAZ_IS_BASE, 0, HW_BAZ_NOOP, 0, 0, HW_BAZ_TRUNCATE, 1, 0};
    }
    // groups: {Label, PulseWidth, StartFrame} 2 bytes, {Pkmax}, {Pkmid}, {Pkmean}, {Pkvar, IsBase} 1 byte each
    __host__ __device__ static constexpr int groupBytes(int i) { return i == 0 ? 2 : (i >= 3 && i <= 6) ? 1 : 0; }
    __host__ __device__ static constexpr bool groupEnd(int i) { return i == 2 || i == 3 || i == 4 || i == 5 || i == 7; }
    __host__ __device__ static constexpr int slot(int) { return 0; }
    __host__ __device__ static constexpr bool skip() { return false; }
    __host__ __device__ static constexpr bool hasDelta() { return true; }
};

// ---- one field: value, transform, serializer ----------------------------------

__device__ __forceinline__ uint64_t RawField(int name, const hw_pulse& p)
{
    return name == HW_BAZ_LABEL ? (uint64_t)p.label
         : name == HW_BAZ_START_FRAME ? (uint64_t)p.start
         : name == HW_BAZ_PULSE_WIDTH ? (uint64_t)p.width
                                      : (uint64_t)(p.is_reject ? 0u : 1u);
}

// Pulse::MaxSignal / MidSignal / MeanSignal / SignalM2 (Pulse.h:105-127):
// fixed-point signals in 0.1 steps, NaN mid signal and M2 below width 3
__device__ __forceinline__ float FloatField(int name, const hw_pulse& p)
{
    const float nan = __int_as_float(0x7fc00000);
    if (name == HW_BAZ_PKMAX) return __fmul_rn((float)p.max_signal, 0.1f);
    if (name == HW_BAZ_PKMID) return p.width < 3 ? nan : __fmul_rn((float)p.mid_signal, 0.1f);
    if (name == HW_BAZ_PKMEAN) return __fmul_rn((float)p.mean_signal, 0.1f);
    return p.width < 3 ? nan : p.signal_m2;
}

// FloatFixedCodec::Apply (FieldTransforms.h:207-251)
__device__ __forceinline__ uint64_t FloatFixed(float v, bool sgn, int scale, int bytes)
{
    float scaled = roundf(__fmul_rn(v, (float)scale));
    if (sgn)
    {
        const int64_t mx = (int64_t)((1ull << (8 * bytes - 1)) - 1 - kFfOffset);
        if ((float)(-mx) <= scaled && (float)mx >= scaled)
        {
            if (scaled >= 0) scaled = __fadd_rn(scaled, (float)kFfOffset);
            return (uint64_t)(int64_t)scaled;
        }
    }
    else
    {
        const uint64_t mx = (1ull << (8 * bytes)) - 1 - kFfOffset;
        if (0 <= scaled && (float)mx >= scaled) return (uint64_t)__fadd_rn(scaled, (float)kFfOffset);
    }
    if (isnan(v)) return kFfNan;
    return scaled < 0 ? kFfNinf : kFfInf;
}

__device__ __forceinline__ uint64_t FieldValue(const hw_baz_field& d, const hw_pulse& p, uint64_t prev)
{
    if (d.transform == HW_BAZ_FLOAT_FIXED)
        return FloatFixed(FloatField(d.name, p), d.store_signed != 0, d.scale, d.transform_bytes);
    const uint64_t raw = RawField(d.name, p);
    return d.transform == HW_BAZ_DELTA ? raw - prev : raw;   // DeltaCompression::Apply
}

__device__ __forceinline__ bool SimpleNeeds(uint64_t v, bool sgn, int bits)
{
    if (sgn) v += (1ull << (bits - 1)) - 1;
    return v >= (1ull << bits) - 1;
}

__device__ __forceinline__ int CompactBytes(uint64_t t, bool sgn, int bits)
{
    if (sgn)
    {
        // leading bits equal to the sign bit, beyond the first
        const uint64_t u = ((int64_t)t < 0) ? ~t : t;
        const int keep = 64 - (__clzll(u) - 1) - (bits - 1);
        return (keep + 6) / 7;
    }
    // 7-bit groups of the bits above the main portion
    const int above = 64 - __clzll(t >> (bits - 1));
    return (above + 6) / 7;
}

__device__ __forceinline__ int OverflowBytes(const hw_baz_field& d, uint64_t v)
{
    if (d.serialize == HW_BAZ_SIMPLE_OVERFLOW) return SimpleNeeds(v, d.store_signed != 0, d.num_bits) ? d.overflow_bytes : 0;
    if (d.serialize == HW_BAZ_COMPACT_OVERFLOW) return CompactBytes(v, d.store_signed != 0, d.num_bits);
    return 0;
}

// Main-portion bits of a field; overflow bytes go to ov (advanced).
__device__ __forceinline__ uint64_t ToBinary(const hw_baz_field& d, uint64_t v, uint8_t*& ov)
{
    const int bits = d.num_bits;
    if (d.serialize == HW_BAZ_SIMPLE_OVERFLOW)
    {
        if (SimpleNeeds(v, d.store_signed != 0, bits))
        {
            for (int b = 0; b < d.overflow_bytes; ++b) ov[b] = (uint8_t)(v >> (8 * b));
            ov += d.overflow_bytes;
            return (1ull << bits) - 1;
        }
        if (d.store_signed) v += (1ull << (bits - 1)) - 1;
        return v;
    }
    if (d.serialize == HW_BAZ_COMPACT_OVERFLOW)
    {
        const uint64_t cmask = 1ull << (bits - 1);
        int n = CompactBytes(v, d.store_signed != 0, bits);
        uint64_t first = v & (cmask - 1);
        v >>= (bits - 1);
        if (n) first |= cmask;
        while (n)
        {
            uint8_t b = (uint8_t)(v & 0x7f);
            v >>= 7;
            --n;
            if (n) b |= 0x80;
            *ov++ = b;
        }
        return first;
    }
    return v;
}

// ---- one pulse -----------------------------------------------------------------

template <class Spec>
__device__ __forceinline__ uint32_t PulseBytes(const Spec& F, const hw_pulse& p, const uint64_t (&prev)[kMaxFields])
{
    uint32_t n = 0;
#pragma unroll
    for (int i = 0; i < kMaxFields; ++i)
    {
        if (i >= F.n()) break;
        const hw_baz_field d = F.f(i);
        n += (uint32_t)F.groupBytes(i) + (uint32_t)OverflowBytes(d, FieldValue(d, p, prev[i]));
    }
    return n;
}

// Groups in order: main bytes little-endian, then the group's overflow bytes
// in field order (ObjectToBaz.h GroupEncoder::Encode).
template <class Spec>
__device__ __forceinline__ uint8_t* EncodePulse(const Spec& F, const hw_pulse& p, const uint64_t (&prev)[kMaxFields],
                                                uint8_t* ptr)
{
    uint64_t data = 0;
    int pos = 0, gBytes = 0;
    uint8_t* main = ptr;
    uint8_t* ov = ptr;
#pragma unroll
    for (int i = 0; i < kMaxFields; ++i)
    {
        if (i >= F.n()) break;
        const hw_baz_field d = F.f(i);
        if (F.groupBytes(i))
        {
            main = ov;
            gBytes = F.groupBytes(i);
            ov = main + gBytes;
            data = 0;
            pos = 0;
        }
        const uint64_t v = ToBinary(d, FieldValue(d, p, prev[i]), ov);
        data |= (v & (uint64_t)((1 << d.num_bits) - 1)) << pos;
        pos += d.num_bits;
        if (F.groupEnd(i))
            for (int b = 0; b < gBytes; ++b) main[b] = (uint8_t)(data >> (8 * b));
    }
    return ov;
}

template <class Spec>
__device__ __forceinline__ void KeepPrev(const Spec& F, const hw_pulse& p, uint64_t (&prev)[kMaxFields])
{
#pragma unroll
    for (int i = 0; i < kMaxFields; ++i)
    {
        if (i >= F.n()) break;
        const hw_baz_field d = F.f(i);
        if (d.transform == HW_BAZ_DELTA) prev[i] = RawField(d.name, p);
    }
}

struct TileArgs
{
    const hw_pulse* pulses;
    const uint32_t* lens;
    uint32_t cap, numZmw, numTiles;
    uint32_t zmwStride;               // ZMWs of a lane encoded: every zmwStride-th
    uint64_t* state;                  // [2][slots][numZmw]; *cur names the copy this call reads
    uint32_t* cur;
    uint64_t* offsets;                // [numZmw + 1]
    uint32_t* events;                 // [numZmw] pulses encoded, or null
    uint8_t* out;
    uint64_t capacity;
    unsigned long long* status;       // [numTiles] look-back words
    unsigned long long* ticket;
    unsigned long long ticketBase;    // the ticket counter's value at launch (0: reset by the call)
    unsigned long long epoch;         // this call's tag in the look-back words
    uint32_t spinLimit;               // polls of a predecessor's word before giving up
    int32_t withhold;                 // tests: this tile never publishes (-1: none)
    volatile uint64_t* host;          // mapped: [0] total bytes, [1] look-back gave up, [2] encoded
};

// look-back words: flag (2 bits) | call epoch (20 bits) | byte count (42 bits)
constexpr int kEpochShift = 42;
constexpr unsigned long long kCountMask = (1ull << kEpochShift) - 1;

__device__ __forceinline__ void StoreRelease(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void StoreRelaxed(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Relaxed: the counts are the only data the tiles exchange, and an acquire
// load would drop the pulses this SM holds in L1.
__device__ __forceinline__ unsigned long long LoadRelaxed(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// The tile's byte count, published as soon as it is known (the first tile's
// is its inclusive total).  Release: the tile read the state-copy word
// before, which the last tile may switch once it has seen every count.
__device__ __forceinline__ void PublishCount(const TileArgs& a, uint32_t tile, uint64_t agg)
{
    const unsigned long long tag = a.epoch << kEpochShift;
    StoreRelease(a.status + tile, (tile == 0 ? kFlagInc : kFlagAgg) | tag | agg);
}

// Decoupled look-back by one warp: sum the counts of the tiles before this
// one back to the nearest one whose inclusive total is known, publish this
// tile's inclusive total.  Words of earlier calls (another epoch) read as
// not ready.  Tiles are taken in ticket order, so every tile waited on has
// started and publishes its count without waiting; the polls are bounded
// all the same.  A tile that gives up, or whose nearest inclusive word is a
// failed one, publishes kFlagFail instead, so every later tile (the call's
// last one included) learns that its prefix is invalid from the status word
// itself; the mapped failure word is written and fenced to system scope
// before that publish.
__device__ uint64_t LookBack(const TileArgs& a, uint32_t tile, uint64_t agg, bool& gaveUp)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long tag = a.epoch << kEpochShift;
    gaveUp = false;
    if (tile == 0 || (int32_t)tile == a.withhold) return 0;
    uint64_t excl = 0;
    int hi = (int)tile - 1;
    uint32_t spins = 0;
    bool failed = false;
    while (true)
    {
        const int idx = hi - lane;
        unsigned long long w = idx >= 0 ? LoadRelaxed(a.status + idx) : (kFlagInc | tag);
        const bool mine = ((w >> kEpochShift) & 0xfffff) == a.epoch;
        const int flag = mine ? (int)(w >> 62) : 0;
        if (__ballot_sync(~0u, flag == 0))
        {
            if ((uint32_t)++spins > a.spinLimit)
            {
                failed = true;
                if (lane == 0)
                {
                    a.host[1] = 1;
                    __threadfence_system();
                }
                break;
            }
            __nanosleep(100);
            continue;
        }
        const uint32_t inc = __ballot_sync(~0u, flag >= 2);
        const int stop = inc ? __ffs(inc) - 1 : 31;
        uint64_t v = lane <= stop ? (w & kCountMask) : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
        excl += v;
        if (inc)
        {
            failed = __shfl_sync(~0u, flag, stop) == 3;
            break;
        }
        hi -= 32;
    }
    gaveUp = failed;
    if (lane == 0) StoreRelaxed(a.status + tile, (failed ? kFlagFail : kFlagInc) | tag | ((excl + agg) & kCountMask));
    return excl;
}

constexpr int kPulseStage = 2048;   // pulses of a tile held in shared memory

// Bytes of shared memory for a tile's encoded bytes (tiles with more are
// written straight to the output); a production pulse is about 2 bytes.
template <class Spec> struct OutStage { static constexpr int bytes = 24 * 1024; };
template <> struct OutStage<ProductionFields> { static constexpr int bytes = 8 * 1024; };

template <class Spec>
constexpr int DynSmem() { return kPulseStage * (int)sizeof(hw_pulse) + OutStage<Spec>::bytes + 32; }

__device__ __forceinline__ void CpAsync4(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}

__device__ __forceinline__ void CpAsync8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}

struct TileView
{
    const TileArgs& a;
    uint32_t z0;
    const uint32_t* rowStart;    // [kTileRows + 1]
    const hw_pulse* pstage;      // the tile's first kPulseStage pulses
    const uint64_t* state0;      // slot 0 of each ZMW's delta state
    const uint64_t* stateCur;
    uint64_t* stateNext;
    // pulse i of the tile, slot k of its ZMW r
    __device__ __forceinline__ hw_pulse At(uint32_t i, int r, int k) const
    {
        return i < (uint32_t)kPulseStage ? pstage[i] : a.pulses[(size_t)(z0 + r) * a.cap + k];
    }
    __device__ __forceinline__ uint64_t State(int slot, int r) const
    {
        return slot == 0 ? state0[r] : stateCur[(size_t)slot * a.numZmw + z0 + r];
    }
};

// One thread's contiguous run of the tile's pulses [i0, i1): sized, with
// the run-relative byte offset of each ZMW starting in it and the delta
// state after each ZMW ending in it (sweep 1), or written at `out` (sweep
// 2).  Returns the run's bytes.
template <class Spec, bool Write>
__device__ __forceinline__ uint32_t Run(const Spec& F, const TileView& t, uint32_t i0, uint32_t i1, uint8_t* out,
                                        uint32_t* rowLocal, uint32_t* rowEvents)
{
    if (i0 >= i1) return 0;
    int lo = 0, hi = kTileRows;   // the ZMW of pulse i0: the last with rowStart <= i0
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (t.rowStart[mid] <= i0) lo = mid; else hi = mid;
    }
    int r = lo, k = (int)(i0 - t.rowStart[lo]);
    uint32_t rowLen = t.rowStart[r + 1] - t.rowStart[r];
    uint64_t prev[kMaxFields];
    if (F.hasDelta())
    {
        // the kept pulse before the run in its ZMW, or the ZMW's state
        int j = k - 1;
        hw_pulse q;
        while (j >= 0)
        {
            q = t.At(i0 - (uint32_t)(k - j), r, j);
            if (!(F.skip() && q.is_reject)) break;
            --j;
        }
#pragma unroll
        for (int f = 0; f < kMaxFields; ++f)
        {
            if (f >= F.n()) break;
            const hw_baz_field d = F.f(f);
            if (d.transform == HW_BAZ_DELTA) prev[f] = j >= 0 ? RawField(d.name, q) : t.State(F.slot(f), r);
        }
    }
    uint32_t bytes = 0, seg = 0;   // seg: pulses kept in this ZMW's part of the run
    for (uint32_t i = i0; i < i1; ++i)
    {
        const hw_pulse p = t.At(i, r, k);
        if (k == 0)
        {
            if (!Write) rowLocal[r] = bytes;
#pragma unroll
            for (int f = 0; f < kMaxFields; ++f)
            {
                if (f >= F.n()) break;
                const hw_baz_field d = F.f(f);
                if (d.transform == HW_BAZ_DELTA) prev[f] = t.State(F.slot(f), r);
            }
        }
        if (!(F.skip() && p.is_reject))
        {
            if (Write) bytes = (uint32_t)(EncodePulse(F, p, prev, out + bytes) - out);
            else bytes += PulseBytes(F, p, prev);
            KeepPrev(F, p, prev);
            ++seg;
        }
        if ((uint32_t)++k == rowLen)
        {
            if (!Write)
            {
                if (seg) atomicAdd(&rowEvents[r], seg);
                // the ZMW's last pulse: the next chunk's delta state (the last
                // kept pulse's values, or the state it came in with)
#pragma unroll
                for (int f = 0; f < kMaxFields; ++f)
                {
                    if (f >= F.n()) break;
                    const hw_baz_field d = F.f(f);
                    if (d.transform == HW_BAZ_DELTA)
                        t.stateNext[(size_t)F.slot(f) * t.a.numZmw + t.z0 + r] = prev[f];
                }
            }
            // the next ZMW with pulses
            do { ++r; } while (r < kTileRows && t.rowStart[r + 1] == t.rowStart[r]);
            k = 0;
            seg = 0;
            rowLen = r < kTileRows ? t.rowStart[r + 1] - t.rowStart[r] : 0;
        }
    }
    if (!Write && seg) atomicAdd(&rowEvents[r], seg);   // the run ends inside a ZMW
    return bytes;
}

template <class Spec>
__global__ void __launch_bounds__(kThreads) BazTileKernel(const __grid_constant__ BazSpec S, const TileArgs a)
{
    using Scan = cub::BlockScan<uint32_t, kThreads>;
    constexpr int kOut = OutStage<Spec>::bytes;
    __shared__ typename Scan::TempStorage scanTmp;
    __shared__ uint32_t rowStart[kTileRows + 1];   // tile pulse index of each ZMW's first pulse
    __shared__ uint32_t rowLocal[kTileRows];       // byte offset of a ZMW's first pulse in its run
    __shared__ uint32_t rowEvents[kTileRows];      // pulses encoded of each ZMW
    __shared__ uint32_t runOffSh[kThreads];        // tile byte offset of each thread's run
    __shared__ uint64_t state0[kTileRows];         // slot 0 of the delta state
    __shared__ uint32_t tileSh, curSh;
    __shared__ uint64_t prefixSh;
    __shared__ int gaveUpSh;
    extern __shared__ __align__(16) uint8_t dyn[];
    hw_pulse* pstage = reinterpret_cast<hw_pulse*>(dyn);
    uint32_t* ostage = reinterpret_cast<uint32_t*>(dyn + kPulseStage * sizeof(hw_pulse));   // then 32 bytes of slack
    const Spec F(S);
    const int tid = threadIdx.x;
    if (tid == 0)
    {
        tileSh = (uint32_t)(atomicAdd(a.ticket, 1ull) - a.ticketBase);
        curSh = *a.cur;
        // the first tile clears the look-back failure word of an earlier call
        // (a tile can only give up long after every tile has started)
        if (tileSh == 0) a.host[1] = 0;
    }
    __syncthreads();
    const uint32_t tile = tileSh;
    const uint32_t z0 = tile * kTileRows;
    const size_t plane = (size_t)(S.slots ? S.slots : 1) * a.numZmw;
    const uint64_t* stateCur = a.state + curSh * plane;
    uint64_t* stateNext = a.state + (1 - curSh) * plane;
    uint32_t cnt = 0;
    if (tid < kTileRows && z0 + tid < a.numZmw && ((z0 + tid) & 63) % a.zmwStride == 0)
        cnt = min(a.lens[z0 + tid], a.cap);   // counts past the slots clamp
    uint32_t excl, P;
    Scan(scanTmp).ExclusiveSum(cnt, excl, P);
    if (tid < kTileRows)
    {
        rowStart[tid] = excl;
        rowEvents[tid] = 0;
        if (z0 + tid < a.numZmw && F.hasDelta()) CpAsync8(&state0[tid], stateCur + z0 + tid);
        if (z0 + tid < a.numZmw && cnt == 0)
        {
            // no pulses this chunk: the state carries over
#pragma unroll
            for (int f = 0; f < kMaxFields; ++f)
            {
                if (f >= F.n()) break;
                const hw_baz_field d = F.f(f);
                if (d.transform != HW_BAZ_DELTA) continue;
                const size_t s = (size_t)F.slot(f) * a.numZmw + z0 + tid;
                stateNext[s] = stateCur[s];
            }
        }
    }
    if (tid == 0) rowStart[kTileRows] = P;
    __syncthreads();
    {
        // the tile's pulses (up to kPulseStage) into shared memory, each
        // warp a ZMW at a time in 4-byte words: 128 contiguous bytes a step
        const int warp = tid >> 5, lane = tid & 31;
        constexpr int kWords = sizeof(hw_pulse) / 4;
        for (int r = warp; r < kTileRows; r += kThreads / 32)
        {
            const uint32_t first = rowStart[r];
            if (first >= (uint32_t)kPulseStage) break;
            const uint32_t n = min(rowStart[r + 1], (uint32_t)kPulseStage) - first;
            const uint32_t* src = reinterpret_cast<const uint32_t*>(a.pulses + (size_t)(z0 + r) * a.cap);
            uint32_t* dst = reinterpret_cast<uint32_t*>(pstage + first);
            for (uint32_t w = lane; w < n * kWords; w += 32) CpAsync4(dst + w, src + w);
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const TileView tv{a, z0, rowStart, pstage, state0, stateCur, stateNext};

    // sweep 1: each thread sizes a contiguous run of the tile's pulses
    const uint32_t per = (P + kThreads - 1) / kThreads;
    const uint32_t i0 = min(P, tid * per), i1 = min(P, i0 + per);
    const uint32_t mine = Run<Spec, false>(F, tv, i0, i1, nullptr, rowLocal, rowEvents);
    uint32_t runOff, tileBytes;
    Scan(scanTmp).ExclusiveSum(mine, runOff, tileBytes);
    runOffSh[tid] = runOff;
    if (tid == 0 && (int32_t)tile != a.withhold) PublishCount(a, tile, tileBytes);
    // sweep 2 into shared memory before the look-back, when the tile fits
    const bool staged = tileBytes <= (uint32_t)kOut;
    if (staged) Run<Spec, true>(F, tv, i0, i1, reinterpret_cast<uint8_t*>(ostage) + runOff, nullptr, nullptr);
    if (tid < 32)
    {
        bool gaveUp;
        const uint64_t prefix = LookBack(a, tile, tileBytes, gaveUp);
        if (tid == 0)
        {
            prefixSh = prefix;
            gaveUpSh = gaveUp;
        }
    }
    __syncthreads();
    const uint64_t prefix = prefixSh;
    const bool fits = prefix + tileBytes <= a.capacity;   // else nothing of this tile is written
    if (fits && staged && tileBytes)
    {
        // out in 16-byte stores at 16-byte boundaries; the two ends, shared
        // with the neighbouring tiles, byte by byte
        const uint32_t mis = (uint32_t)(reinterpret_cast<uintptr_t>(a.out + prefix) & 15);
        uint8_t* base = a.out + prefix - mis;
        const uint32_t end = mis + tileBytes;
        const uint8_t* sb = reinterpret_cast<const uint8_t*>(ostage);
        for (uint32_t lo = tid * 16; lo < end; lo += kThreads * 16)
        {
            if (lo >= mis && lo + 16 <= end)
            {
                const uint32_t src = lo - mis, w = src >> 2, sh = (src & 3) * 8;
                const uint32_t x0 = ostage[w], x1 = ostage[w + 1], x2 = ostage[w + 2], x3 = ostage[w + 3],
                               x4 = ostage[w + 4];
                uint4 v;
                v.x = __funnelshift_r(x0, x1, sh);
                v.y = __funnelshift_r(x1, x2, sh);
                v.z = __funnelshift_r(x2, x3, sh);
                v.w = __funnelshift_r(x3, x4, sh);
                *reinterpret_cast<uint4*>(base + lo) = v;
            }
            else
            {
                for (uint32_t b = max(lo, mis); b < min(lo + 16, end); ++b) base[b] = sb[b - mis];
            }
        }
    }
    else if (fits && !staged)
    {
        Run<Spec, true>(F, tv, i0, i1, a.out + prefix + runOff, nullptr, nullptr);
    }

    if (tid < kTileRows && z0 + tid < a.numZmw)
    {
        // a ZMW without pulses starts where the next one with pulses does
        int r = tid;
        while (r < kTileRows && rowStart[r] == rowStart[r + 1]) ++r;
        a.offsets[z0 + tid] = prefix + (r < kTileRows ? runOffSh[rowStart[r] / per] + rowLocal[r] : tileBytes);
        if (a.events) a.events[z0 + tid] = rowEvents[tid];
    }
    if (tile == a.numTiles - 1 && tid == 0)
    {
        // every tile read *cur before it published its count, and every
        // count has been seen
        __threadfence();
        const uint64_t total = prefix + tileBytes;
        const bool ok = total <= a.capacity && !gaveUpSh && a.host[1] == 0;
        a.offsets[a.numZmw] = total;
        a.host[0] = total;
        a.host[2] = ok ? 1 : 0;
        if (ok) *a.cur = 1 - curSh;
    }
}

int Fail(int code, const std::string& msg) { return hwk::SetLastError(code, msg.c_str()); }

int CheckFields(const hw_baz_field* f, uint32_t n)
{
    if (!f || n == 0 || n > (uint32_t)kMaxFields) return Fail(HW_ERR_INVALID_ARG, "BAZ encoding: 1 to 16 fields");
    for (uint32_t i = 0; i < n; ++i)
    {
        const hw_baz_field& d = f[i];
        if (d.name < HW_BAZ_LABEL || d.name > HW_BAZ_PKVAR || d.num_bits < 1 || d.num_bits > 30 ||
            d.serialize < HW_BAZ_TRUNCATE || d.serialize > HW_BAZ_COMPACT_OVERFLOW || d.transform < HW_BAZ_NOOP ||
            d.transform > HW_BAZ_FLOAT_FIXED)
            return Fail(HW_ERR_INVALID_ARG, "BAZ encoding: bad field");
        const bool isFloat = d.name >= HW_BAZ_PKMAX;
        if (isFloat != (d.transform == HW_BAZ_FLOAT_FIXED))
            return Fail(HW_ERR_INVALID_ARG, "BAZ encoding: signal fields need the fixed-point codec, others an integer transform");
        // 8-byte codes are left out: a float of 2^63 or 2^64 passes the range
        // check and its conversion to an integer is undefined
        if (d.transform == HW_BAZ_FLOAT_FIXED && (d.transform_bytes < 1 || d.transform_bytes > 7 || d.scale < 1))
            return Fail(HW_ERR_INVALID_ARG, "BAZ encoding: fixed-point codes of 1 to 7 bytes");
        // a signed compact field of more than 14 bits would count a negative
        // number of overflow bytes for small values (FieldSerializers.h CompactOverflow)
        if (d.serialize == HW_BAZ_COMPACT_OVERFLOW && d.store_signed && d.num_bits > 14)
            return Fail(HW_ERR_INVALID_ARG, "BAZ encoding: signed compact fields of at most 14 bits");
        if (d.serialize == HW_BAZ_SIMPLE_OVERFLOW && (d.overflow_bytes < 1 || d.overflow_bytes > 8))
            return Fail(HW_ERR_INVALID_ARG, "BAZ encoding: bad overflow size");
    }
    return HW_OK;
}

// Does the list equal a constant one (same fields, groups and reject rule)?
template <class Spec>
bool SameAs(const BazSpec& S)
{
    if (S.n != Spec::n() || (S.skipRejects != 0) != Spec::skip()) return false;
    for (int i = 0; i < S.n; ++i)
    {
        const hw_baz_field a = S.f[i], b = Spec::f(i);
        if (a.name != b.name || a.store_signed != b.store_signed || a.transform != b.transform ||
            a.serialize != b.serialize || a.num_bits != b.num_bits ||
            (a.transform == HW_BAZ_FLOAT_FIXED && (a.scale != b.scale || a.transform_bytes != b.transform_bytes)) ||
            (a.serialize == HW_BAZ_SIMPLE_OVERFLOW && a.overflow_bytes != b.overflow_bytes) ||
            S.groupBytes[i] != Spec::groupBytes(i) || (S.groupEnd[i] != 0) != Spec::groupEnd(i) ||
            (a.transform == HW_BAZ_DELTA && S.slot[i] != Spec::slot(i)))
            return false;
    }
    return true;
}

}   // namespace

struct hw_baz_encoder
{
    BazSpec spec{};
    int kind = 0;                  // 0 runtime list, 1 production, 2 internal
    uint32_t numZmw = 0, numTiles = 0, zmwStride = 1;
    uint64_t* state = nullptr;     // [2][slots][numZmw] delta state
    uint32_t* cur = nullptr;       // device: the state copy the next call reads
    unsigned long long* status = nullptr;   // [numTiles] look-back words, then the ticket counter
    unsigned long long epoch = 0;           // the last call's tag (20 bits; 0 never used)
    uint32_t spinLimit = kSpinLimit;        // look-back polls before a tile gives up
    int32_t withhold = -1;                  // tests: a tile that never publishes
    uint64_t* host = nullptr;      // mapped pinned words
    uint64_t* hostDev = nullptr;
    ~hw_baz_encoder() { cudaFree(state); cudaFree(status); cudaFreeHost(host); }
};

namespace {

template <class Spec>
cudaError_t Launch(uint32_t tiles, const BazSpec& spec, const TileArgs& a, cudaStream_t s)
{
    static std::atomic<uint64_t> devicesSet{0};   // the shared memory above 48 KB, set once a device
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return ce;
    const uint64_t bit = 1ull << (dev & 63);
    if (!(devicesSet.load() & bit))
    {
        ce = cudaFuncSetAttribute(BazTileKernel<Spec>, cudaFuncAttributeMaxDynamicSharedMemorySize, DynSmem<Spec>());
        if (ce != cudaSuccess) return ce;
        devicesSet.fetch_or(bit);
    }
    (void)cudaGetLastError();   // an earlier, unrelated failure is not this launch's
    BazTileKernel<Spec><<<tiles, kThreads, DynSmem<Spec>(), s>>>(spec, a);
    return cudaGetLastError();
}

// Enqueues one chunk's encoding.
int Enqueue(hw_baz_encoder* e, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
            uint8_t* d_bytes, uint64_t bytes_capacity, uint64_t* d_offsets, uint32_t* d_events, cudaStream_t s)
{
    if (!d_bytes) bytes_capacity = 0;
    cudaError_t ce = cudaSuccess;
    if (++e->epoch == (1ull << 20))
    {
        // the tags wrap: clear the words so no word of an old call reads as this one's
        ce = cudaMemsetAsync(e->status, 0, sizeof(unsigned long long) * e->numTiles, s);
        e->epoch = 1;
    }
    // tickets count from 0 every call, whatever became of earlier launches
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e->status + e->numTiles, 0, sizeof(unsigned long long), s);
    TileArgs a;
    a.pulses = d_pulses;
    a.lens = d_lens;
    a.cap = max_calls;
    a.numZmw = e->numZmw;
    a.numTiles = e->numTiles;
    a.zmwStride = e->zmwStride;
    a.state = e->state;
    a.cur = e->cur;
    a.offsets = d_offsets;
    a.events = d_events;
    a.out = d_bytes;
    a.capacity = bytes_capacity;
    a.status = e->status;
    a.ticket = e->status + e->numTiles;
    a.ticketBase = 0;
    a.epoch = e->epoch;
    a.spinLimit = e->spinLimit;
    a.withhold = e->withhold;
    a.host = e->hostDev;
    if (ce == cudaSuccess)
    {
        if (e->kind == 1) ce = Launch<ProductionFields>(e->numTiles, e->spec, a, s);
        else if (e->kind == 2) ce = Launch<InternalFields>(e->numTiles, e->spec, a, s);
        else ce = Launch<RtFields>(e->numTiles, e->spec, a, s);
    }
    if (ce != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_baz_encode: ") + cudaGetErrorString(ce));
    return HW_OK;
}

int Result(hw_baz_encoder* e, uint64_t* total_bytes)
{
    volatile uint64_t* h = e->host;
    *total_bytes = h[0];
    if (h[1]) return Fail(HW_ERR_TIMEOUT, "hw_baz_encode: a tile's look-back gave up waiting");
    if (!h[2]) return Fail(HW_ERR_OUT_OF_MEMORY, "hw_baz_encode: the chunk needs more than bytes_capacity");
    return HW_OK;
}

}   // namespace

extern "C" {

int hw_baz_preset(int32_t which, hw_baz_field* fields, uint32_t* n_fields, int32_t* skip_rejects)
{
    if (!fields || !n_fields || (which != 0 && which != 1)) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    const int n = which == 0 ? ProductionFields::n() : InternalFields::n();
    for (int i = 0; i < n; ++i) fields[i] = which == 0 ? ProductionFields::f(i) : InternalFields::f(i);
    *n_fields = (uint32_t)n;
    if (skip_rejects) *skip_rejects = which == 0 ? 1 : 0;   // PrelimHQFilter.cpp:116
    return HW_OK;
}

int hw_baz_encoder_create(const hw_baz_field* fields, uint32_t n_fields, int32_t skip_rejects, uint32_t num_zmw,
                          hw_baz_encoder** out)
{
    if (!out || num_zmw == 0) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    *out = nullptr;
    int rc = CheckFields(fields, n_fields);
    if (rc) return rc;
    auto e = new hw_baz_encoder;
    e->numZmw = num_zmw;
    e->numTiles = (num_zmw + kTileRows - 1) / kTileRows;
    BazSpec& S = e->spec;
    S.n = (int)n_fields;
    S.skipRejects = skip_rejects != 0;
    // grouping (ObjectToBaz.h:373-393): close the group when it is a whole,
    // non-zero number of bytes or the next field would pass 64 bits
    int cur = 0, open = -1;
    for (uint32_t i = 0; i < n_fields; ++i)
    {
        S.f[i] = fields[i];
        const int bits = fields[i].num_bits;
        if (open < 0 || (cur % 8 == 0 && cur > 0) || cur + bits > 64)
        {
            if (open >= 0)
            {
                S.groupEnd[i - 1] = 1;
                S.groupBytes[open] = (cur + 7) / 8;
            }
            open = (int)i;
            cur = 0;
        }
        cur += bits;
        if (fields[i].transform == HW_BAZ_DELTA) S.slot[i] = S.slots++;
    }
    S.groupEnd[n_fields - 1] = 1;
    S.groupBytes[open] = (cur + 7) / 8;
    e->kind = SameAs<ProductionFields>(S) ? 1 : SameAs<InternalFields>(S) ? 2 : 0;
    const size_t stateBytes = sizeof(uint64_t) * 2 * (size_t)(S.slots ? S.slots : 1) * num_zmw;
    cudaError_t ce = cudaMalloc((void**)&e->state, stateBytes + sizeof(uint64_t));
    if (ce == cudaSuccess) ce = cudaMemset(e->state, 0, stateBytes + sizeof(uint64_t));
    if (ce == cudaSuccess) e->cur = reinterpret_cast<uint32_t*>(e->state + stateBytes / sizeof(uint64_t));
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->status, sizeof(unsigned long long) * (e->numTiles + 1));
    if (ce == cudaSuccess) ce = cudaMemset(e->status, 0, sizeof(unsigned long long) * (e->numTiles + 1));
    if (ce == cudaSuccess) ce = cudaHostAlloc((void**)&e->host, 4 * sizeof(uint64_t), cudaHostAllocMapped);
    if (ce == cudaSuccess)
        for (int i = 0; i < 4; ++i) e->host[i] = 0;   // pinned memory comes uninitialised
    if (ce == cudaSuccess) ce = cudaHostGetDevicePointer((void**)&e->hostDev, e->host, 0);
    if (ce != cudaSuccess)
    {
        delete e;
        return Fail(HW_ERR_CUDA, std::string("hw_baz_encoder_create: ") + cudaGetErrorString(ce));
    }
    *out = e;
    return HW_OK;
}

int hw_baz_encoder_destroy(hw_baz_encoder* e)
{
    delete e;
    return HW_OK;
}

int hw_baz_encoder_set_wait_limit(hw_baz_encoder* e, uint32_t polls, int32_t withhold_tile)
{
    if (!e || polls == 0) return Fail(HW_ERR_INVALID_ARG, "hw_baz_encoder_set_wait_limit: bad argument");
    e->spinLimit = polls;
    e->withhold = withhold_tile;
    return HW_OK;
}

int hw_baz_encoder_set_zmw_stride(hw_baz_encoder* e, uint32_t stride)
{
    if (!e || stride == 0 || 64 % stride != 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_baz_encoder_set_zmw_stride: the stride must divide 64");
    e->zmwStride = stride;
    return HW_OK;
}

int hw_baz_encode(hw_baz_encoder* e, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                  uint8_t* d_bytes, uint64_t bytes_capacity, uint64_t* d_offsets, uint32_t* d_events,
                  uint64_t* total_bytes, void* stream)
{
    const NvtxRange range("hw_baz_encode");
    if (!e || !d_pulses || !d_lens || !d_offsets || !total_bytes || max_calls == 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_baz_encode: bad argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int rc = Enqueue(e, d_pulses, d_lens, max_calls, d_bytes, bytes_capacity, d_offsets, d_events, s);
    if (rc) return rc;
    const cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_baz_encode: ") + cudaGetErrorString(ce));
    return Result(e, total_bytes);
}

int hw_baz_encode_async(hw_baz_encoder* e, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                        uint8_t* d_bytes, uint64_t bytes_capacity, uint64_t* d_offsets, uint32_t* d_events,
                        void* stream)
{
    if (!e || !d_pulses || !d_lens || !d_offsets || max_calls == 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_baz_encode_async: bad argument");
    return Enqueue(e, d_pulses, d_lens, max_calls, d_bytes, bytes_capacity, d_offsets, d_events,
                   reinterpret_cast<cudaStream_t>(stream));
}

int hw_baz_encode_result(hw_baz_encoder* e, uint64_t* total_bytes)
{
    if (!e || !total_bytes) return Fail(HW_ERR_INVALID_ARG, "hw_baz_encode_result: bad argument");
    return Result(e, total_bytes);
}

}   // extern "C"
