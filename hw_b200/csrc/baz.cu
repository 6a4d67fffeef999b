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
// One thread per ZMW.  Pass 1 sizes every ZMW's bytes for the chunk (on a
// copy of its delta state), an exclusive scan places the ZMWs one after the
// other, pass 2 encodes each ZMW's pulses at its offset and advances the
// state.
#include <string>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "hw_device.cuh"

using namespace hwk;

namespace {

constexpr int kMaxFields = 16;
constexpr uint64_t kFfNan = 0, kFfInf = 1, kFfNinf = 2, kFfOffset = 3;   // FloatFixedCodec codes

struct BazSpec
{
    hw_baz_field f[kMaxFields];
    int groupEnd[kMaxFields];     // 1: the field closes its group
    int groupBytes[kMaxFields];   // nominal bytes of the group a field opens (0 elsewhere)
    int n;
    int skipRejects;
};

struct BazPulseVals
{
    uint32_t label, start, width, isBase;
    float pkmax, pkmid, pkmean, pkvar;
};

__device__ __forceinline__ BazPulseVals Values(const hw_pulse& p)
{
    const float nan = __int_as_float(0x7fc00000);
    BazPulseVals v;
    v.label = p.label;
    v.start = p.start;
    v.width = p.width;
    v.isBase = p.is_reject ? 0u : 1u;
    v.pkmax = __fmul_rn((float)p.max_signal, 0.1f);
    v.pkmid = p.width < 3 ? nan : __fmul_rn((float)p.mid_signal, 0.1f);
    v.pkmean = __fmul_rn((float)p.mean_signal, 0.1f);
    v.pkvar = p.width < 3 ? nan : p.signal_m2;
    return v;
}

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

// Transformed value of field i; the delta state of the field advances.
__device__ __forceinline__ uint64_t FieldValue(const hw_baz_field& d, const BazPulseVals& p, uint64_t& last)
{
    if (d.transform == HW_BAZ_FLOAT_FIXED)
    {
        const float v = d.name == HW_BAZ_PKMAX ? p.pkmax : d.name == HW_BAZ_PKMID ? p.pkmid
                      : d.name == HW_BAZ_PKMEAN ? p.pkmean : p.pkvar;
        return FloatFixed(v, d.store_signed != 0, d.scale, d.transform_bytes);
    }
    const uint64_t raw = d.name == HW_BAZ_LABEL ? p.label : d.name == HW_BAZ_START_FRAME ? p.start
                       : d.name == HW_BAZ_PULSE_WIDTH ? p.width : p.isBase;
    if (d.transform == HW_BAZ_DELTA)
    {
        const uint64_t r = raw - last;
        last = raw;
        return r;
    }
    return raw;
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
        const int discard = __clzll(u) - 1;
        const int keep = 64 - discard - (bits - 1);
        return (keep + 6) / 7;
    }
    t >>= (bits - 1);
    int r = 0;
    while (t) { ++r; t >>= 7; }
    return r;
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

__device__ __forceinline__ int PulseBytes(const BazSpec& S, const BazPulseVals& p, uint64_t* last)
{
    int n = 0;
    for (int i = 0; i < S.n; ++i) n += S.groupBytes[i] + OverflowBytes(S.f[i], FieldValue(S.f[i], p, last[i]));
    return n;
}

__device__ __forceinline__ uint8_t* EncodePulse(const BazSpec& S, const BazPulseVals& p, uint8_t* ptr, uint64_t* last)
{
    uint64_t data = 0;
    int pos = 0, gBytes = 0;
    uint8_t* main = ptr;
    uint8_t* ov = ptr;
    for (int i = 0; i < S.n; ++i)
    {
        if (S.groupBytes[i])
        {
            // a new group: main bytes first, overflow bytes after them
            main = ov;
            gBytes = S.groupBytes[i];
            ov = main + gBytes;
            data = 0;
            pos = 0;
        }
        const int bits = S.f[i].num_bits;
        const uint64_t v = ToBinary(S.f[i], FieldValue(S.f[i], p, last[i]), ov);
        data |= (v & (uint64_t)((1 << bits) - 1)) << pos;
        pos += bits;
        if (S.groupEnd[i])
            for (int b = 0; b < gBytes; ++b) main[b] = (uint8_t)(data >> (8 * b));
    }
    return ov;
}

// Pass 1: offsets[z] = the bytes of ZMW z this chunk (on a copy of its
// delta state); offsets[numZmw] = 0, so the exclusive scan that follows
// leaves the total there.
__global__ void BazSizeKernel(BazSpec S, const hw_pulse* pulses, const uint32_t* lens, int cap, int numZmw,
                              const uint64_t* state, uint64_t* offsets)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z == 0) offsets[numZmw] = 0;
    if (z >= numZmw) return;
    uint64_t last[kMaxFields];
    for (int i = 0; i < S.n; ++i) last[i] = state[(size_t)z * kMaxFields + i];
    uint64_t bytes = 0;
    const hw_pulse* row = pulses + (size_t)z * cap;
    const uint32_t n = min(lens[z], (uint32_t)cap);   // counts past the slots are clamped
    for (uint32_t k = 0; k < n; ++k)
    {
        const hw_pulse p = row[k];
        if (S.skipRejects && p.is_reject) continue;
        bytes += (uint64_t)PulseBytes(S, Values(p), last);
    }
    offsets[z] = bytes;
}

// Pass 2: each ZMW's pulses at its offset; the delta state advances.  When
// the chunk needs more than `capacity` bytes nothing is written and the
// state stays.  The total goes to the mapped host word.
__global__ void BazEncodeKernel(BazSpec S, const hw_pulse* pulses, const uint32_t* lens, int cap, int numZmw,
                                uint64_t* state, const uint64_t* offsets, uint8_t* out, uint64_t capacity,
                                volatile uint64_t* hostTotal)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t total = offsets[numZmw];
    if (z == 0) *hostTotal = total;
    if (z >= numZmw || total > capacity) return;
    uint64_t last[kMaxFields];
    for (int i = 0; i < S.n; ++i) last[i] = state[(size_t)z * kMaxFields + i];
    uint8_t* ptr = out + offsets[z];
    const hw_pulse* row = pulses + (size_t)z * cap;
    const uint32_t n = min(lens[z], (uint32_t)cap);   // counts past the slots are clamped
    for (uint32_t k = 0; k < n; ++k)
    {
        const hw_pulse p = row[k];
        if (S.skipRejects && p.is_reject) continue;
        ptr = EncodePulse(S, Values(p), ptr, last);
    }
    for (int i = 0; i < S.n; ++i) state[(size_t)z * kMaxFields + i] = last[i];
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

}   // namespace

struct hw_baz_encoder
{
    BazSpec spec{};
    uint32_t numZmw = 0;
    uint64_t* state = nullptr;     // [numZmw][kMaxFields] delta state
    void* scanTmp = nullptr;
    size_t scanTmpBytes = 0;
    uint64_t* hostTotal = nullptr;  // mapped pinned word
    uint64_t* devTotal = nullptr;   // its device address
    ~hw_baz_encoder() { cudaFree(state); cudaFree(scanTmp); cudaFreeHost(hostTotal); }
};

extern "C" {

int hw_baz_preset(int32_t which, hw_baz_field* fields, uint32_t* n_fields, int32_t* skip_rejects)
{
    if (!fields || !n_fields || (which != 0 && which != 1)) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    // PulseGroups.h:42-53 ProductionPulses, :55-94 InternalPulses
    const hw_baz_field label{HW_BAZ_LABEL, 0, HW_BAZ_NOOP, 0, 0, HW_BAZ_TRUNCATE, 2, 0};
    const hw_baz_field width{HW_BAZ_PULSE_WIDTH, 0, HW_BAZ_NOOP, 0, 0, HW_BAZ_COMPACT_OVERFLOW, 7, 0};
    const hw_baz_field start{HW_BAZ_START_FRAME, 0, HW_BAZ_DELTA, 0, 0, HW_BAZ_COMPACT_OVERFLOW, 7, 0};
    uint32_t n = 0;
    fields[n++] = label;
    fields[n++] = width;
    fields[n++] = start;
    if (which == 1)
    {
        fields[n++] = hw_baz_field{HW_BAZ_PKMAX, 1, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 8, 2};
        fields[n++] = hw_baz_field{HW_BAZ_PKMID, 1, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 8, 2};
        fields[n++] = hw_baz_field{HW_BAZ_PKMEAN, 1, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 8, 2};
        fields[n++] = hw_baz_field{HW_BAZ_PKVAR, 0, HW_BAZ_FLOAT_FIXED, 10, 2, HW_BAZ_SIMPLE_OVERFLOW, 7, 2};
        fields[n++] = hw_baz_field{HW_BAZ_IS_BASE, 0, HW_BAZ_NOOP, 0, 0, HW_BAZ_TRUNCATE, 1, 0};
    }
    *n_fields = n;
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
    }
    S.groupEnd[n_fields - 1] = 1;
    S.groupBytes[open] = (cur + 7) / 8;
    cudaError_t ce = cudaMalloc((void**)&e->state, sizeof(uint64_t) * kMaxFields * num_zmw);
    if (ce == cudaSuccess) ce = cudaMemset(e->state, 0, sizeof(uint64_t) * kMaxFields * num_zmw);
    if (ce == cudaSuccess) ce = cudaHostAlloc((void**)&e->hostTotal, sizeof(uint64_t), cudaHostAllocMapped);
    if (ce == cudaSuccess) ce = cudaHostGetDevicePointer((void**)&e->devTotal, e->hostTotal, 0);
    if (ce == cudaSuccess)
        ce = cub::DeviceScan::ExclusiveSum(nullptr, e->scanTmpBytes, e->state, e->state, (int)num_zmw + 1);
    if (ce == cudaSuccess) ce = cudaMalloc(&e->scanTmp, e->scanTmpBytes);
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

int hw_baz_encode(hw_baz_encoder* e, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                  uint8_t* d_bytes, uint64_t bytes_capacity, uint64_t* d_offsets, uint64_t* total_bytes,
                  void* stream)
{
    if (!e || !d_pulses || !d_lens || !d_offsets || !total_bytes || max_calls == 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_baz_encode: bad argument");
    if (!d_bytes) bytes_capacity = 0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int n = (int)e->numZmw;
    const int threads = 128, blocks = (n + threads - 1) / threads;
    BazSizeKernel<<<blocks, threads, 0, s>>>(e->spec, d_pulses, d_lens, (int)max_calls, n, e->state, d_offsets);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess)
        ce = cub::DeviceScan::ExclusiveSum(e->scanTmp, e->scanTmpBytes, d_offsets, d_offsets, n + 1, s);
    if (ce == cudaSuccess)
    {
        BazEncodeKernel<<<blocks, threads, 0, s>>>(e->spec, d_pulses, d_lens, (int)max_calls, n, e->state, d_offsets,
                                                   d_bytes, bytes_capacity, e->devTotal);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_baz_encode: ") + cudaGetErrorString(ce));
    const uint64_t total = *(volatile uint64_t*)e->hostTotal;
    *total_bytes = total;
    if (total > bytes_capacity)
        return Fail(HW_ERR_OUT_OF_MEMORY, "hw_baz_encode: the chunk needs more than bytes_capacity");
    return HW_OK;
}

}   // extern "C"
