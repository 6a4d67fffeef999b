// Learned DME initializer: a 302 -> 256 -> 256 -> 19 MLP (BF16 weights and
// activations, FP32 accumulation, GELU) that proposes the EM start of each
// ZMW from its trace histogram and baseline statistics.  No counterpart in
// the reference: the reference always starts its EM from PrelimEstimate and
// ScaleModelSnr (DmeEmHost.cpp:161-361); hw_dme_em_fit runs the EM from the
// proposal and falls back to that plain start when the proposal's
// log-likelihood is lower.
//
// Layout.  Samples are rows: features [n][304] (302 used), outputs and
// targets [n][32] (19 used).  Weights are stored [out][in] (row-major), so
// every GEMM of the forward pass reads both operands along K, the layout of
// mma.sync's row.col BF16 tensor-core instruction.  The GEMM stages tiles of
// either operand, in any of its strides, through shared memory as BF16, so
// the same kernel serves the backward products (X^T dZ, dZ W).
#include <cuda_bf16.h>

#include "hw_device.cuh"

namespace hwk {

constexpr int kFeat = 304;          // 300 bins + baseline mean + variance, padded to a multiple of 16
constexpr int kHidden = 256;
constexpr int kOut = 32;            // 19 outputs, padded
constexpr int kOutUsed = 19;

// Parameter layout (floats): W1 [256][304], b1 [256], W2 [256][256], b2 [256],
// W3 [32][256], b3 [32].  Rows 19..31 of W3 and b3 stay 0.
constexpr size_t kOffW1 = 0;
constexpr size_t kOffB1 = kOffW1 + (size_t)kHidden * kFeat;
constexpr size_t kOffW2 = kOffB1 + kHidden;
constexpr size_t kOffB2 = kOffW2 + (size_t)kHidden * kHidden;
constexpr size_t kOffW3 = kOffB2 + kHidden;
constexpr size_t kOffB3 = kOffW3 + (size_t)kOut * kHidden;
constexpr size_t kParams = kOffB3 + kOut;

// ---- features, targets, proposals -------------------------------------------

// Per ZMW: sqrt of each bin's share of the in-range counts, then the baseline
// mean (in bins above the histogram's low bound) and variance (in squared
// bins) of the baseliner statistics.  Everything is in units of the
// histogram's own bin size, which the histogram reset ties to the baseline
// sigma, so the features do not depend on the trace's offset or gain.
// One CTA of 256 threads per lane: the first 64 threads reduce the per-ZMW
// totals, then the lane's 64 x 304 features are written row after row, so
// consecutive threads write consecutive addresses.
constexpr int kFeatThreads = 256;

// Per ZMW: the inverse of the in-range count total and the two baseline
// features (shared by the features kernel and the fused proposal).
__device__ __forceinline__ void FeatureRow(const hw_lane_histogram& H, const hw_baseliner_stats& st, int z,
                                           float& inv, float& fMean, float& fVar)
{
    // the integer total (below 2^24 for any histogram the accumulator fills,
    // so equal to the float sum in any order)
    uint32_t count = 0;
    for (int b = 0; b < kBins; ++b) count += H.bin_count[b][z];
    const float total = (float)count;
    inv = total > 0.0f ? 1.0f / total : 0.0f;
    const float lb = H.low_bound[z], bs = H.bin_size[z];
    const hw_stat_accum_state& S = st.baseline_stats;
    const float m0 = S.moment0[z], m1 = S.moment1[z], m2 = S.moment2[z];
    const float mean = m0 > 0.0f ? m1 / m0 + S.offset[z] : lb;
    const float var = m0 > 1.0f ? fmaxf((m2 - m1 * m1 / m0) / (m0 - 1.0f), 0.0f) : bs * bs;
    const float fm = (mean - lb) / bs, fv = var / (bs * bs);
    fMean = isfinite(fm) ? fm : 0.0f;
    fVar = isfinite(fv) ? fv : 0.0f;
}

__device__ __forceinline__ float FeatureValue(const hw_lane_histogram& H, int z, int b, float inv, float fMean,
                                              float fVar)
{
    if (b < kBins) return sqrtf((float)H.bin_count[b][z] * inv);
    if (b == kBins) return fMean;
    if (b == kBins + 1) return fVar;
    return 0.0f;
}

__global__ void __launch_bounds__(kFeatThreads) FeaturesKernel(const hw_lane_histogram* __restrict__ hist,
                                                               const hw_baseliner_stats* __restrict__ st,
                                                               float* __restrict__ out)
{
    const int l = blockIdx.x, tid = threadIdx.x;
    const hw_lane_histogram& H = hist[l];
    __shared__ float inv[kLane], fMean[kLane], fVar[kLane];
    if (tid < kLane) FeatureRow(H, st[l], tid, inv[tid], fMean[tid], fVar[tid]);
    __syncthreads();
    float* f = out + (size_t)l * kLane * kFeat;
    for (int e = tid; e < kLane * kFeat; e += kFeatThreads)
    {
        const int z = e / kFeat, b = e % kFeat;
        f[e] = FeatureValue(H, z, b, inv[z], fMean[z], fVar[z]);
    }
}

// Training targets from fitted EM parameters params [lanes][15][64]:
// 0 baseline mean (bins above the low bound), 1 log baseline variance
// (squared bins), 2-5 analog means, 6-9 log analog variances, 10-14 mixture
// fractions, 15-18 the analogs' excess-noise terms (XsnCoeffCVSq,
// DetectionModelHost.cpp:248-256); 19-31 are 0.
__global__ void TargetsKernel(const float* __restrict__ params, const hw_lane_histogram* __restrict__ hist,
                              float shotVarCoeff, float* __restrict__ out)
{
    const int l = blockIdx.x, z = threadIdx.x;
    const float* P = params + (size_t)l * 15 * kLane;
    const float lb = hist[l].low_bound[z], bs = hist[l].bin_size[z];
    float* t = out + ((size_t)l * kLane + z) * kOut;
    auto rho = [&](int i) { return P[i * kLane + z]; };
    auto mu = [&](int i) { return P[(5 + i) * kLane + z]; };
    auto var = [&](int i) { return P[(10 + i) * kLane + z]; };
    t[0] = (mu(0) - lb) / bs;
    t[1] = logf(fmaxf(var(0), 1e-6f) / (bs * bs));
    for (int a = 0; a < 4; ++a)
    {
        t[2 + a] = (mu(a + 1) - lb) / bs;
        t[6 + a] = logf(fmaxf(var(a + 1), 1e-6f) / (bs * bs));
        const float m = mu(a + 1);
        t[15 + a] = ((var(a + 1) - var(0)) - shotVarCoeff * m) / fmaxf(m * m, 1e-6f);
    }
    for (int i = 0; i < 5; ++i) t[10 + i] = rho(i);
    for (int i = kOutUsed; i < kOut; ++i) t[i] = 0.0f;
}

// EM start from network outputs y [n][32] (standardised; mean/scale undo
// the standardisation): the inverse of TargetsKernel, with fractions floored
// at 0.001 and renormalised and variances floored at 1e-3 squared bins.
__device__ __forceinline__ void ProposalFromOutputs(const float* Y, const float* __restrict__ mean,
                                                    const float* __restrict__ scale, float lb, float bs, float* P,
                                                    int z)
{
    auto o = [&](int i) { return Y[i] * scale[i] + mean[i]; };
    float rs = 0.0f, r[5];
    for (int i = 0; i < 5; ++i) { r[i] = fmaxf(o(10 + i), 0.001f); rs += r[i]; }
    for (int i = 0; i < 5; ++i) P[i * kLane + z] = r[i] / rs;
    P[5 * kLane + z] = lb + o(0) * bs;
    P[10 * kLane + z] = bs * bs * fmaxf(expf(fminf(o(1), 30.0f)), 1e-3f);
    for (int a = 0; a < 4; ++a)
    {
        P[(6 + a) * kLane + z] = lb + o(2 + a) * bs;
        P[(11 + a) * kLane + z] = bs * bs * fmaxf(expf(fminf(o(6 + a), 30.0f)), 1e-3f);
    }
}

__global__ void ProposalKernel(const float* __restrict__ y, const float* __restrict__ mean,
                               const float* __restrict__ scale, const hw_lane_histogram* __restrict__ hist,
                               float* __restrict__ proposal)
{
    const int l = blockIdx.x, z = threadIdx.x;
    ProposalFromOutputs(y + ((size_t)l * kLane + z) * kOut, mean, scale, hist[l].low_bound[z], hist[l].bin_size[z],
                        proposal + (size_t)l * 15 * kLane, z);
}

// ---- BF16 tensor-core GEMM ----------------------------------------------------
// C[m][n] = sum_k A(m,k) B(k,n), A(m,k) = A[m*sam + k*sak], B(k,n) =
// B[k*sbk + n*sbn], sources float or bf16 (converted to bf16 when staged).
// Epilogue kStore: C = result; kBiasGelu: Z = result + bias[n] stored to C,
// GELU(Z) stored as bf16 to H[m*shm + n]; kBias: C = result + bias[n].
enum GemmEpilogue { kStore = 0, kBiasGelu = 1, kBias = 2 };

constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;

template <typename T> __device__ __forceinline__ __nv_bfloat16 ToBf16(T v);
template <> __device__ __forceinline__ __nv_bfloat16 ToBf16<float>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 ToBf16<__nv_bfloat16>(__nv_bfloat16 v) { return v; }

__device__ __forceinline__ float GeluTanh(float x)
{
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}

__device__ __forceinline__ float GeluTanhGrad(float x)
{
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    const float t = tanhf(k0 * (x + k1 * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k0 * (1.0f + 3.0f * k1 * x * x);
}

__device__ __forceinline__ uint32_t Pack2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(128) GemmKernel(const TA* __restrict__ A, long sam, long sak,
                                                  const TB* __restrict__ B, long sbk, long sbn, float* __restrict__ C,
                                                  long scm, int M, int N, int K, int epilogue,
                                                  const float* __restrict__ bias, __nv_bfloat16* __restrict__ H,
                                                  long shm)
{
    __shared__ __nv_bfloat16 sA[kBM][kBK + kPad];      // [m][k]
    __shared__ __nv_bfloat16 sB[kBN][kBK + kPad];      // [n][k]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;     // warp tile 32 x 32
    const int g = lane >> 2, q = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[i][j][c] = 0.0f;

    for (int k0 = 0; k0 < K; k0 += kBK)
    {
        for (int e = tid; e < kBM * kBK; e += 128)
        {
            const int r = e / kBK, c = e % kBK;
            const int m = m0 + r, k = k0 + c;
            sA[r][c] = (m < M && k < K) ? ToBf16(A[(long)m * sam + (long)k * sak]) : __float2bfloat16_rn(0.0f);
        }
        for (int e = tid; e < kBN * kBK; e += 128)
        {
            const int r = e / kBK, c = e % kBK;
            const int n = n0 + r, k = k0 + c;
            sB[r][c] = (n < N && k < K) ? ToBf16(B[(long)k * sbk + (long)n * sbn]) : __float2bfloat16_rn(0.0f);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16)
        {
            uint32_t af[2][4], bfr[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
            {
                const int r = wm + i * 16 + g;
                af[i][0] = Pack2(sA[r][kk + 2 * q], sA[r][kk + 2 * q + 1]);
                af[i][1] = Pack2(sA[r + 8][kk + 2 * q], sA[r + 8][kk + 2 * q + 1]);
                af[i][2] = Pack2(sA[r][kk + 2 * q + 8], sA[r][kk + 2 * q + 9]);
                af[i][3] = Pack2(sA[r + 8][kk + 2 * q + 8], sA[r + 8][kk + 2 * q + 9]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int n = wn + j * 8 + g;
                bfr[j][0] = Pack2(sB[n][kk + 2 * q], sB[n][kk + 2 * q + 1]);
                bfr[j][1] = Pack2(sB[n][kk + 2 * q + 8], sB[n][kk + 2 * q + 9]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                        : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                        : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bfr[j][0]),
                          "r"(bfr[j][1]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                const int m = m0 + wm + i * 16 + g + (c >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + 2 * q + (c & 1);
                if (m >= M || n >= N) continue;
                float v = acc[i][j][c];
                if (epilogue != kStore) v += bias[n];
                C[(long)m * scm + n] = v;
                if (epilogue == kBiasGelu) H[(long)m * shm + n] = __float2bfloat16_rn(GeluTanh(v));
            }
}

// ---- Fused forward pass on the sm_100 tensor cores (tcgen05 + TMEM) ------------
// One CTA of 128 threads per 128 rows runs all three layers: the
// standardised BF16 input tile and each layer's BF16 weights are staged in
// shared memory as canonical K-major core matrices (8 rows x 16 bytes,
// no swizzle: rows 16 bytes apart, the next 8-column group 128 bytes on,
// the next 8-row group K * 16 bytes on); one thread issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, K = 16 a step) into a
// 256-column FP32 accumulator in tensor memory and commits to an mbarrier;
// the four warps read their 32 rows back (tcgen05.ld 32x32b), add the bias,
// apply GELU and write the BF16 activations over the input tile as the next
// layer's A operand.  Layer 1 runs as two N = 128 halves so that a weight
// half (76 KB) and the input tile (76 KB) fit beside each other; layer 2
// takes all of W2 (128 KB).  Rounding points are those of the mma.sync
// path (BF16 inputs and activations, FP32 accumulation and epilogue); only
// the order of the FP32 accumulation differs.  Every wait on the mbarrier
// is bounded: past about a second the CTA writes NaN rows (a proposal the
// DME's fallback test rejects), sets *err and returns.
constexpr int kTcRows = 128;
constexpr int kTcThreads = 512;        // 16 warps: warp w reads TMEM lanes 32 (w % 4) .. + 31
constexpr uint32_t kTcCols = 256;                                      // TMEM columns
constexpr int kTcA = kTcRows * kFeat * 2;                             // 77,824 B: input tile, then activations
constexpr int kTcW = kHidden * kHidden * 2;                           // 131,072 B: the largest weight block
constexpr int kTcSmem = kTcA + kTcW;

__device__ __forceinline__ uint32_t SmemU32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no-swizzle UMMA shared-memory descriptor (sm_100 version bit 46).
__device__ __forceinline__ uint64_t UmmaDesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128.
__host__ __device__ constexpr uint32_t UmmaIdesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void UmmaBf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 :: "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}

__device__ __forceinline__ bool MbarTryWait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// All threads: wait for the MMAs committed to `bar` (phase `parity`); false
// (for every thread) when any thread gave up.
__device__ __forceinline__ bool WaitMmas(uint32_t bar, uint32_t parity)
{
    const long long t0 = clock64();
    bool ok = false;
    while (!(ok = MbarTryWait(bar, parity)))
        if (clock64() - t0 > 4000000000ll) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return !__syncthreads_or(!ok);
}

// Issued by one thread: D[tmem] (+)= A (128 x K) . B (N x K)^T over K / 16 steps.
__device__ __forceinline__ void MmaChain(uint32_t d, uint32_t a, uint32_t b, int k, int n, uint32_t bar)
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t sbo = (uint32_t)k * 16u, idesc = UmmaIdesc(n);
    for (int s = 0; s < k / 16; ++s)
        UmmaBf16(d, UmmaDesc(a + s * 256u, 128u, sbo), UmmaDesc(b + s * 256u, 128u, sbo), idesc, s > 0);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar)
                 : "memory");
}

// Byte offset of 16-byte chunk c (columns 8c..8c+7) of row r in a K-column tile.
__device__ __forceinline__ uint32_t CoreOffset(int r, int c, int k)
{
    return (uint32_t)((r >> 3) * k * 16 + c * 128 + (r & 7) * 16);
}

// rows x k BF16 weights (row stride k) into the canonical layout, 32 bytes a task.
__device__ __forceinline__ void StageWeights(const __nv_bfloat16* __restrict__ w, int rows, int k, uint8_t* dst)
{
    const int pairs = k / 16;
    for (int t = threadIdx.x; t < rows * pairs; t += kTcThreads)
    {
        const int r8 = t & 7, rest = t >> 3, c2 = rest % pairs, g = rest / pairs, r = g * 8 + r8;
        const uint4* src = reinterpret_cast<const uint4*>(w + (size_t)r * k + c2 * 16);
        const uint4 lo = __ldg(src), hi = __ldg(src + 1);
        *reinterpret_cast<uint4*>(dst + CoreOffset(r, 2 * c2, k)) = lo;
        *reinterpret_cast<uint4*>(dst + CoreOffset(r, 2 * c2 + 1, k)) = hi;
    }
}

// The standardised input tile (rows past n are 0), as InputKernel rounds it.
__device__ __forceinline__ void StageInput(const float* __restrict__ feat, long row0, long n,
                                           const float* __restrict__ mean, const float* __restrict__ scale,
                                           uint8_t* dst)
{
    const int pairs = kFeat / 16;
    for (int t = threadIdx.x; t < kTcRows * pairs; t += kTcThreads)
    {
        const int r8 = t & 7, rest = t >> 3, c2 = rest % pairs, g = rest / pairs, r = g * 8 + r8;
        uint32_t packed[8];
        if (row0 + r < n)
        {
            const float4* src = reinterpret_cast<const float4*>(feat + (row0 + r) * kFeat + c2 * 16);
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const float4 v = __ldg(src + q);
                const int c = c2 * 16 + q * 4;
                const __nv_bfloat16 a = __float2bfloat16_rn((v.x - mean[c]) / scale[c]);
                const __nv_bfloat16 b = __float2bfloat16_rn((v.y - mean[c + 1]) / scale[c + 1]);
                const __nv_bfloat16 e = __float2bfloat16_rn((v.z - mean[c + 2]) / scale[c + 2]);
                const __nv_bfloat16 f = __float2bfloat16_rn((v.w - mean[c + 3]) / scale[c + 3]);
                packed[2 * q] = Pack2(a, b);
                packed[2 * q + 1] = Pack2(e, f);
            }
        }
        else
        {
#pragma unroll
            for (int q = 0; q < 8; ++q) packed[q] = 0;
        }
        *reinterpret_cast<uint4*>(dst + CoreOffset(r, 2 * c2, kFeat)) =
            make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *reinterpret_cast<uint4*>(dst + CoreOffset(r, 2 * c2 + 1, kFeat)) =
            make_uint4(packed[4], packed[5], packed[6], packed[7]);
    }
}

// The same tile computed from the lanes' histograms and baseliner statistics
// (FeatureRow / FeatureValue, as FeaturesKernel): rows are ZMWs of the lanes
// row0 / 64 and the next.
__device__ __forceinline__ void StageInputFromHist(const hw_lane_histogram* __restrict__ hist,
                                                   const hw_baseliner_stats* __restrict__ st, long row0, long n,
                                                   const float* __restrict__ mean, const float* __restrict__ scale,
                                                   uint8_t* dst, float* rowInv, float* rowMean, float* rowVar)
{
    if (threadIdx.x < kTcRows)
    {
        const long row = row0 + threadIdx.x;
        if (row < n)
            FeatureRow(hist[row / kLane], st[row / kLane], (int)(row % kLane), rowInv[threadIdx.x],
                       rowMean[threadIdx.x], rowVar[threadIdx.x]);
    }
    __syncthreads();
    const int pairs = kFeat / 16;
    for (int t = threadIdx.x; t < kTcRows * pairs; t += kTcThreads)
    {
        const int r8 = t & 7, rest = t >> 3, c2 = rest % pairs, g = rest / pairs, r = g * 8 + r8;
        uint32_t packed[8];
        const long row = row0 + r;
        if (row < n)
        {
            const hw_lane_histogram& H = hist[row / kLane];
            const int z = (int)(row % kLane);
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                const int c = c2 * 16 + 2 * q;
                const float f0 = FeatureValue(H, z, c, rowInv[r], rowMean[r], rowVar[r]);
                const float f1 = FeatureValue(H, z, c + 1, rowInv[r], rowMean[r], rowVar[r]);
                packed[q] = Pack2(__float2bfloat16_rn((f0 - mean[c]) / scale[c]),
                                  __float2bfloat16_rn((f1 - mean[c + 1]) / scale[c + 1]));
            }
        }
        else
        {
#pragma unroll
            for (int q = 0; q < 8; ++q) packed[q] = 0;
        }
        *reinterpret_cast<uint4*>(dst + CoreOffset(r, 2 * c2, kFeat)) =
            make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *reinterpret_cast<uint4*>(dst + CoreOffset(r, 2 * c2 + 1, kFeat)) =
            make_uint4(packed[4], packed[5], packed[6], packed[7]);
    }
}

// Generic-proxy shared-memory writes made visible to the tensor cores, then a
// CTA barrier (with the TMEM reads before it ordered).
__device__ __forceinline__ void PublishShared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
}

// 32 accumulator columns [col, col + 32) of this thread's row.
__device__ __forceinline__ void TmemLoad32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Hidden-layer epilogue: bias, GELU, BF16 into the A tile (K = 256 layout).
// Warp w takes row 32 (w % 4) + lane, columns 64 (w / 4) .. + 63.
__device__ __forceinline__ void HiddenEpilogue(uint32_t tbase, const float* __restrict__ bias, uint8_t* a)
{
    const int warp = threadIdx.x >> 5, quad = warp & 3, r = quad * 32 + (threadIdx.x & 31);
    for (int c0 = (warp >> 2) * 64; c0 < (warp >> 2) * 64 + 64; c0 += 32)
    {
        float v[32];
        TmemLoad32(tbase + ((uint32_t)(quad * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            uint32_t p[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int c = c0 + q * 8 + 2 * j;
                const float z0 = v[q * 8 + 2 * j] + bias[c], z1 = v[q * 8 + 2 * j + 1] + bias[c + 1];
                p[j] = Pack2(__float2bfloat16_rn(GeluTanh(z0)), __float2bfloat16_rn(GeluTanh(z1)));
            }
            *reinterpret_cast<uint4*>(a + CoreOffset(r, c0 / 8 + q, kHidden)) = make_uint4(p[0], p[1], p[2], p[3]);
        }
    }
}

struct TcArgs
{
    const float* feat;                 // [n][304] features, or
    const hw_lane_histogram* hist;     // the lanes' histograms and statistics (n = lanes * 64)
    const hw_baseliner_stats* stats;
    long n;
    const float* inMean;
    const float* inScale;
    const float* outMean;
    const float* outScale;
    const __nv_bfloat16* wb;
    const float* master;
    float* out;                        // [n][32] standardised outputs, or
    float* proposal;                   // [lanes][15][64] EM starts
    int* err;
};

// kHist: features from the histograms and the proposal written directly.
template <bool kHist>
__global__ void __launch_bounds__(kTcThreads, 1) ForwardTcKernel(TcArgs p)
{
    extern __shared__ __align__(1024) uint8_t tcSmem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmemSlot;
    __shared__ float rowInv[kTcRows], rowMean[kTcRows], rowVar[kTcRows];
    const long n = p.n;
    const __nv_bfloat16* __restrict__ wb = p.wb;
    const float* __restrict__ master = p.master;
    uint8_t* A = tcSmem;
    uint8_t* W = tcSmem + kTcA;
    const uint32_t aAddr = SmemU32(A), wAddr = SmemU32(W), barAddr = SmemU32(&bar);
    const int warp = threadIdx.x >> 5;
    const long row0 = (long)blockIdx.x * kTcRows;
    // the output rows: warps 0..3, one row a thread
    const bool outWarp = warp < 4;
    const long myRow = row0 + (threadIdx.x & (kTcRows - 1));

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(SmemU32(&tmemSlot)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(barAddr) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (kHist) StageInputFromHist(p.hist, p.stats, row0, n, p.inMean, p.inScale, A, rowInv, rowMean, rowVar);
    else StageInput(p.feat, row0, n, p.inMean, p.inScale, A);
    StageWeights(wb + kOffW1, kHidden / 2, kFeat, W);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    PublishShared();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tmemSlot;

    bool ok = true;
    uint32_t parity = 0;
    // layer 1, columns 0..127 then 128..255
    for (int half = 0; half < 2 && ok; ++half)
    {
        if (half)
        {
            StageWeights(wb + kOffW1 + (size_t)(kHidden / 2) * kFeat, kHidden / 2, kFeat, W);
            PublishShared();
        }
        if (threadIdx.x == 0) MmaChain(tbase + (uint32_t)(half * 128), aAddr, wAddr, kFeat, 128, barAddr);
        ok = WaitMmas(barAddr, parity);
        parity ^= 1;
    }
    // layer 2
    if (ok)
    {
        HiddenEpilogue(tbase, master + kOffB1, A);
        StageWeights(wb + kOffW2, kHidden, kHidden, W);
        PublishShared();
        if (threadIdx.x == 0) MmaChain(tbase, aAddr, wAddr, kHidden, kHidden, barAddr);
        ok = WaitMmas(barAddr, parity);
        parity ^= 1;
    }
    // layer 3
    if (ok)
    {
        HiddenEpilogue(tbase, master + kOffB2, A);
        StageWeights(wb + kOffW3, kOut, kHidden, W);
        PublishShared();
        if (threadIdx.x == 0) MmaChain(tbase, aAddr, wAddr, kHidden, kOut, barAddr);
        ok = WaitMmas(barAddr, parity);
    }
    if (ok && outWarp)
    {
        float v[32];
        TmemLoad32(tbase + ((uint32_t)(warp * 32) << 16), v);
        const float* b3 = master + kOffB3;
#pragma unroll
        for (int q = 0; q < kOut; ++q) v[q] = v[q] + b3[q];
        if (myRow < n)
        {
            if (kHist)
            {
                const long l = myRow / kLane;
                const int z = (int)(myRow % kLane);
                ProposalFromOutputs(v, p.outMean, p.outScale, p.hist[l].low_bound[z], p.hist[l].bin_size[z],
                                    p.proposal + l * 15 * kLane, z);
            }
            else
            {
                float4* o = reinterpret_cast<float4*>(p.out + myRow * kOut);
#pragma unroll
                for (int q = 0; q < kOut / 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
    }
    else if (!ok)
    {
        if (threadIdx.x == 0) atomicCAS(p.err, 0, HW_ERR_TIMEOUT);
        if (outWarp && myRow < n)
        {
            const float nan = __int_as_float(0x7fc00000);
            if (kHist)
                for (int q = 0; q < 15; ++q) p.proposal[(myRow / kLane) * 15 * kLane + q * kLane + myRow % kLane] = nan;
            else
                for (int q = 0; q < kOut; ++q) p.out[myRow * kOut + q] = nan;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tbase), "r"(kTcCols) : "memory");
}

// ---- training helpers ---------------------------------------------------------

// Network input: rows idx[i] (or i) of the features, standardised, as bf16.
__global__ void InputKernel(const float* __restrict__ feat, const int32_t* __restrict__ idx, int n,
                            const float* __restrict__ mean, const float* __restrict__ scale,
                            __nv_bfloat16* __restrict__ X)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)n * kFeat) return;
    const int i = (int)(e / kFeat), c = (int)(e % kFeat);
    const long row = idx ? idx[i] : i;
    X[e] = __float2bfloat16_rn((feat[row * kFeat + c] - mean[c]) / scale[c]);
}

// Standardised targets of rows idx[i] (or i); unused columns are 0.
__global__ void TargetGatherKernel(const float* __restrict__ tgt, const int32_t* __restrict__ idx, int n,
                                   const float* __restrict__ mean, const float* __restrict__ scale,
                                   float* __restrict__ T)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * kOut) return;
    const int i = e / kOut, c = e % kOut;
    const long row = idx ? idx[i] : i;
    T[e] = c < kOutUsed ? (tgt[row * kOut + c] - mean[c]) / scale[c] : 0.0f;
}

// Mean squared error over the 19 used outputs: dY = 2 (Y - T) / (n * 19);
// the loss is accumulated into *loss.
__global__ void LossGradKernel(const float* __restrict__ Y, const float* __restrict__ T, int n,
                               float* __restrict__ dY, float* __restrict__ loss)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (e < n * kOut)
    {
        const int c = e % kOut;
        const float d = c < kOutUsed ? Y[e] - T[e] : 0.0f;
        const float inv = 1.0f / ((float)n * (float)kOutUsed);
        dY[e] = 2.0f * d * inv;
        l = d * d * inv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// dZ = dH * GELU'(Z), elementwise (may run in place on dH).
__global__ void GeluBackKernel(const float* __restrict__ dH, const float* __restrict__ Z, long count,
                               float* __restrict__ dZ)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < count) dZ[e] = dH[e] * GeluTanhGrad(Z[e]);
}

// Column sums of D [n][cols] (bias gradients), one thread per column.
__global__ void ColSumKernel(const float* __restrict__ D, int n, int cols, float* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += D[(long)i * cols + c];
    out[c] = s;
}

// AdamW (decoupled weight decay) on FP32 master parameters; refreshes the
// BF16 copy when one is given.
__global__ void AdamWKernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int count, float lr, float b1, float b2, float eps, float wd,
                            float c1, float c2, __nv_bfloat16* __restrict__ wb)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.0f - b1) * gi;
    const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    const float mh = mi / c1, vh = vi / c2;
    const float wi = w[e] - lr * (mh / (sqrtf(vh) + eps) + wd * w[e]);
    w[e] = wi;
    if (wb) wb[e] = __float2bfloat16_rn(wi);
}

__global__ void ToBf16Kernel(const float* __restrict__ src, int count, __nv_bfloat16* __restrict__ dst)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < count) dst[e] = __float2bfloat16_rn(src[e]);
}

}   // namespace hwk

// ---- handle and C ABI -----------------------------------------------------------

#include <random>
#include <vector>

namespace {

using namespace hwk;

int Cuda(cudaError_t e, const char* where)
{
    if (e == cudaSuccess) return HW_OK;
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return SetLastError(e == cudaErrorMemoryAllocation ? HW_ERR_OUT_OF_MEMORY : HW_ERR_CUDA, m.c_str());
}

template <typename TA, typename TB>
cudaError_t Gemm(const TA* A, long sam, long sak, const TB* B, long sbk, long sbn, float* C, long scm, int M, int N,
                 int K, int epi, const float* bias, __nv_bfloat16* H, long shm, cudaStream_t s)
{
    const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
    GemmKernel<TA, TB><<<grid, 128, 0, s>>>(A, sam, sak, B, sbk, sbn, C, scm, M, N, K, epi, bias, H, shm);
    return cudaGetLastError();
}

inline unsigned Blocks(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}   // namespace

struct hw_learned_init
{
    uint32_t maxBatch = 0;
    int step = 0;
    float* master = nullptr;   // FP32 parameters
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    __nv_bfloat16* wb = nullptr;   // BF16 copy of all parameters (the weight blocks are used)
    float* norm = nullptr;     // input mean [304], input scale [304], output mean [32], output scale [32]
    __nv_bfloat16* X = nullptr;
    float* Z1 = nullptr;
    __nv_bfloat16* H1 = nullptr;
    float* Z2 = nullptr;
    __nv_bfloat16* H2 = nullptr;
    float* Y = nullptr;
    float* T = nullptr;
    float* dY = nullptr;
    float* dA = nullptr;       // [maxBatch][256] hidden gradient
    float* loss = nullptr;
    int* err = nullptr;        // set by the tensor-core forward pass when a wait timed out

    float* InMean() const { return norm; }
    float* InScale() const { return norm + kFeat; }
    float* OutMean() const { return norm + 2 * kFeat; }
    float* OutScale() const { return norm + 2 * kFeat + kOut; }

    ~hw_learned_init()
    {
        cudaFree(master); cudaFree(grad); cudaFree(m); cudaFree(v); cudaFree(wb); cudaFree(norm);
        cudaFree(X); cudaFree(Z1); cudaFree(H1); cudaFree(Z2); cudaFree(H2); cudaFree(Y); cudaFree(T);
        cudaFree(dY); cudaFree(dA); cudaFree(loss); cudaFree(err);
    }

    // The fused tensor-core forward pass over a.n rows.
    template <bool kHist>
    int LaunchTc(TcArgs a, cudaStream_t s, const char* where)
    {
        static bool attr = false;
        if (!attr)
        {
            const int rc = Cuda(cudaFuncSetAttribute(ForwardTcKernel<kHist>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     kTcSmem), where);
            if (rc) return rc;
            attr = true;
        }
        a.inMean = InMean();
        a.inScale = InScale();
        a.outMean = OutMean();
        a.outScale = OutScale();
        a.wb = wb;
        a.master = master;
        a.err = err;
        ForwardTcKernel<kHist><<<(unsigned)((a.n + kTcRows - 1) / kTcRows), kTcThreads, kTcSmem, s>>>(a);
        return Cuda(cudaGetLastError(), where);
    }

    // Forward pass of n <= maxBatch rows (rows idx[i], or i, of feat): outputs in Y.
    cudaError_t Forward(const float* feat, const int32_t* idx, int n, cudaStream_t s)
    {
        InputKernel<<<Blocks((long)n * kFeat), 256, 0, s>>>(feat, idx, n, InMean(), InScale(), X);
        cudaError_t e = cudaGetLastError();
        if (e) return e;
        if ((e = Gemm(X, kFeat, 1, wb + kOffW1, 1, kFeat, Z1, kHidden, n, kHidden, kFeat, kBiasGelu,
                      master + kOffB1, H1, kHidden, s))) return e;
        if ((e = Gemm(H1, kHidden, 1, wb + kOffW2, 1, kHidden, Z2, kHidden, n, kHidden, kHidden, kBiasGelu,
                      master + kOffB2, H2, kHidden, s))) return e;
        return Gemm(H2, kHidden, 1, wb + kOffW3, 1, kHidden, Y, kOut, n, kOut, kHidden, kBias, master + kOffB3,
                    (__nv_bfloat16*)nullptr, 0, s);
    }

    // Loss and gradients (into grad) of n rows; the loss is added to *loss.
    cudaError_t Backward(const float* tgt, const int32_t* idx, int n, cudaStream_t s)
    {
        TargetGatherKernel<<<Blocks((long)n * kOut), 256, 0, s>>>(tgt, idx, n, OutMean(), OutScale(), T);
        LossGradKernel<<<Blocks((long)n * kOut), 256, 0, s>>>(Y, T, n, dY, loss);
        cudaError_t e = cudaGetLastError();
        if (e) return e;
        // layer 3: dW3 = dY^T H2, db3 = colsum dY, dH2 = dY W3
        if ((e = Gemm(dY, 1, kOut, H2, kHidden, 1, grad + kOffW3, kHidden, kOut, kHidden, n, kStore,
                      (const float*)nullptr, (__nv_bfloat16*)nullptr, 0, s))) return e;
        ColSumKernel<<<1, kOut, 0, s>>>(dY, n, kOut, grad + kOffB3);
        if ((e = Gemm(dY, kOut, 1, wb + kOffW3, kHidden, 1, dA, kHidden, n, kHidden, kOut, kStore,
                      (const float*)nullptr, (__nv_bfloat16*)nullptr, 0, s))) return e;
        GeluBackKernel<<<Blocks((long)n * kHidden), 256, 0, s>>>(dA, Z2, (long)n * kHidden, dA);
        // layer 2: dW2 = dZ2^T H1, db2, dH1 = dZ2 W2
        if ((e = Gemm(dA, 1, kHidden, H1, kHidden, 1, grad + kOffW2, kHidden, kHidden, kHidden, n, kStore,
                      (const float*)nullptr, (__nv_bfloat16*)nullptr, 0, s))) return e;
        ColSumKernel<<<1, kHidden, 0, s>>>(dA, n, kHidden, grad + kOffB2);
        // dH1 goes to Z2's buffer (Z2 is no longer needed)
        if ((e = Gemm(dA, kHidden, 1, wb + kOffW2, kHidden, 1, Z2, kHidden, n, kHidden, kHidden, kStore,
                      (const float*)nullptr, (__nv_bfloat16*)nullptr, 0, s))) return e;
        GeluBackKernel<<<Blocks((long)n * kHidden), 256, 0, s>>>(Z2, Z1, (long)n * kHidden, dA);
        // layer 1: dW1 = dZ1^T X, db1
        if ((e = Gemm(dA, 1, kHidden, X, kFeat, 1, grad + kOffW1, kFeat, kHidden, kFeat, n, kStore,
                      (const float*)nullptr, (__nv_bfloat16*)nullptr, 0, s))) return e;
        ColSumKernel<<<1, kHidden, 0, s>>>(dA, n, kHidden, grad + kOffB1);
        return cudaGetLastError();
    }
};

extern "C" {

int hw_learned_init_create(uint32_t max_batch, uint64_t seed, hw_learned_init** out)
{
    if (!out || max_batch == 0 || max_batch > (1u << 20))
        return SetLastError(HW_ERR_INVALID_ARG, "hw_learned_init_create: max_batch must be in [1, 2^20]");
    *out = nullptr;
    auto h = new hw_learned_init();
    h->maxBatch = max_batch;
    const size_t B = max_batch;
    int rc = HW_OK;
    auto alloc = [&](auto** p, size_t count) {
        if (rc == HW_OK) rc = Cuda(cudaMalloc((void**)p, count * sizeof(**p)), "hw_learned_init_create");
    };
    alloc(&h->master, kParams); alloc(&h->grad, kParams); alloc(&h->m, kParams); alloc(&h->v, kParams);
    alloc(&h->wb, kParams); alloc(&h->norm, 2 * kFeat + 2 * kOut);
    alloc(&h->X, B * kFeat); alloc(&h->Z1, B * kHidden); alloc(&h->H1, B * kHidden); alloc(&h->Z2, B * kHidden);
    alloc(&h->H2, B * kHidden); alloc(&h->Y, B * kOut); alloc(&h->T, B * kOut); alloc(&h->dY, B * kOut);
    alloc(&h->dA, B * kHidden); alloc(&h->loss, 1); alloc(&h->err, 1);
    if (!rc) rc = Cuda(cudaMemset(h->err, 0, sizeof(int)), "hw_learned_init_create");
    if (rc) { delete h; return rc; }
    // He-normal weights (std sqrt(2 / fan_in)) from a seeded host generator,
    // zero biases, zero rows for the unused outputs.
    std::vector<float> w(kParams, 0.0f);
    std::mt19937_64 gen(seed);
    auto fill = [&](size_t off, int rows, int cols) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)cols));
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) w[off + (size_t)r * cols + c] = nd(gen);
    };
    fill(kOffW1, kHidden, kFeat);
    fill(kOffW2, kHidden, kHidden);
    fill(kOffW3, kOutUsed, kHidden);
    std::vector<float> norm(2 * kFeat + 2 * kOut, 0.0f);
    for (int i = 0; i < kFeat; ++i) norm[kFeat + i] = 1.0f;
    for (int i = 0; i < kOut; ++i) norm[2 * kFeat + kOut + i] = 1.0f;
    if (!rc) rc = Cuda(cudaMemcpy(h->master, w.data(), kParams * 4, cudaMemcpyHostToDevice), "hw_learned_init_create");
    if (!rc) rc = Cuda(cudaMemcpy(h->norm, norm.data(), norm.size() * 4, cudaMemcpyHostToDevice), "hw_learned_init_create");
    if (!rc) rc = Cuda(cudaMemset(h->m, 0, kParams * 4), "hw_learned_init_create");
    if (!rc) rc = Cuda(cudaMemset(h->v, 0, kParams * 4), "hw_learned_init_create");
    if (!rc) rc = Cuda(cudaMemset(h->grad, 0, kParams * 4), "hw_learned_init_create");
    if (!rc)
    {
        ToBf16Kernel<<<Blocks((long)kParams), 256>>>(h->master, (int)kParams, h->wb);
        rc = Cuda(cudaDeviceSynchronize(), "hw_learned_init_create");
    }
    if (rc) { delete h; return rc; }
    *out = h;
    return HW_OK;
}

int hw_learned_init_destroy(hw_learned_init* h)
{
    delete h;
    return HW_OK;
}

int hw_learned_init_param_count(uint32_t* count)
{
    if (!count) return SetLastError(HW_ERR_INVALID_ARG, "count is NULL");
    *count = (uint32_t)kParams;
    return HW_OK;
}

int hw_learned_init_get_params(const hw_learned_init* h, float* host_params, float* host_norm)
{
    if (!h) return SetLastError(HW_ERR_INVALID_ARG, "NULL handle");
    int rc = HW_OK;
    if (host_params) rc = Cuda(cudaMemcpy(host_params, h->master, kParams * 4, cudaMemcpyDeviceToHost), "get_params");
    if (!rc && host_norm)
        rc = Cuda(cudaMemcpy(host_norm, h->norm, (2 * kFeat + 2 * kOut) * 4, cudaMemcpyDeviceToHost), "get_params");
    return rc;
}

int hw_learned_init_set_params(hw_learned_init* h, const float* host_params, const float* host_norm)
{
    if (!h) return SetLastError(HW_ERR_INVALID_ARG, "NULL handle");
    int rc = HW_OK;
    if (host_params)
    {
        rc = Cuda(cudaMemcpy(h->master, host_params, kParams * 4, cudaMemcpyHostToDevice), "set_params");
        if (!rc)
        {
            ToBf16Kernel<<<Blocks((long)kParams), 256>>>(h->master, (int)kParams, h->wb);
            rc = Cuda(cudaDeviceSynchronize(), "set_params");
        }
    }
    if (!rc && host_norm)
        rc = Cuda(cudaMemcpy(h->norm, host_norm, (2 * kFeat + 2 * kOut) * 4, cudaMemcpyHostToDevice), "set_params");
    return rc;
}

int hw_learned_init_features(uint32_t lanes, const hw_lane_histogram* d_hist, const hw_baseliner_stats* d_stats,
                             float* d_features, void* stream)
{
    if (!d_hist || !d_stats || !d_features || lanes == 0) return SetLastError(HW_ERR_INVALID_ARG, "bad argument");
    FeaturesKernel<<<lanes, kFeatThreads, 0, (cudaStream_t)stream>>>(d_hist, d_stats, d_features);
    return Cuda(cudaGetLastError(), "hw_learned_init_features");
}

int hw_learned_init_targets(const hw_config* cfg, uint32_t lanes, const float* d_params,
                            const hw_lane_histogram* d_hist, float* d_targets, void* stream)
{
    if (!cfg || !d_params || !d_hist || !d_targets || lanes == 0) return SetLastError(HW_ERR_INVALID_ARG, "bad argument");
    TargetsKernel<<<lanes, kLane, 0, (cudaStream_t)stream>>>(d_params, d_hist, cfg->shot_var_coeff, d_targets);
    return Cuda(cudaGetLastError(), "hw_learned_init_targets");
}

int hw_learned_init_forward(hw_learned_init* h, const float* d_features, uint32_t n, float* d_out, void* stream)
{
    if (!h || !d_features || !d_out) return SetLastError(HW_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return HW_OK;
    TcArgs a{};
    a.feat = d_features;
    a.n = n;
    a.out = d_out;
    return h->LaunchTc<false>(a, (cudaStream_t)stream, "hw_learned_init_forward");
}

int hw_learned_init_propose(hw_learned_init* h, uint32_t lanes, const hw_lane_histogram* d_hist,
                            const hw_baseliner_stats* d_stats, float* d_proposal, void* stream)
{
    if (!h || !d_hist || !d_stats || !d_proposal) return SetLastError(HW_ERR_INVALID_ARG, "bad argument");
    if (lanes == 0) return HW_OK;
    TcArgs a{};
    a.hist = d_hist;
    a.stats = d_stats;
    a.n = (long)lanes * kLane;
    a.proposal = d_proposal;
    return h->LaunchTc<true>(a, (cudaStream_t)stream, "hw_learned_init_propose");
}

int hw_learned_init_forward_status(hw_learned_init* h)
{
    if (!h) return SetLastError(HW_ERR_INVALID_ARG, "bad argument");
    int e = 0;
    int rc = Cuda(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost), "hw_learned_init_forward_status");
    if (rc) return rc;
    if (e)
    {
        cudaMemset(h->err, 0, sizeof(int));
        return SetLastError(e, "hw_learned_init_forward: a tensor-core wait timed out (rows written as NaN)");
    }
    return HW_OK;
}

int hw_learned_init_proposal(const hw_learned_init* h, uint32_t lanes, const float* d_out,
                             const hw_lane_histogram* d_hist, float* d_proposal, void* stream)
{
    if (!h || !d_out || !d_hist || !d_proposal || lanes == 0) return SetLastError(HW_ERR_INVALID_ARG, "bad argument");
    ProposalKernel<<<lanes, kLane, 0, (cudaStream_t)stream>>>(d_out, h->OutMean(), h->OutScale(), d_hist, d_proposal);
    return Cuda(cudaGetLastError(), "hw_learned_init_proposal");
}

// Gradients of the mean squared error of n <= max_batch rows (rows d_index[i],
// or i, of the features and raw targets) into the handle; optionally copied to
// d_grad.  Synchronous: *loss receives the loss.
int hw_learned_init_gradients(hw_learned_init* h, const float* d_features, const float* d_targets,
                              const int32_t* d_index, uint32_t n, float* d_grad, float* loss, void* stream)
{
    if (!h || !d_features || !d_targets || n == 0 || n > h->maxBatch)
        return SetLastError(HW_ERR_INVALID_ARG, "hw_learned_init_gradients: 1 <= n <= max_batch");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = Cuda(cudaMemsetAsync(h->loss, 0, 4, s), "hw_learned_init_gradients");
    if (!rc) rc = Cuda(h->Forward(d_features, d_index, (int)n, s), "hw_learned_init_gradients");
    if (!rc) rc = Cuda(h->Backward(d_targets, d_index, (int)n, s), "hw_learned_init_gradients");
    if (!rc && d_grad)
        rc = Cuda(cudaMemcpyAsync(d_grad, h->grad, kParams * 4, cudaMemcpyDeviceToDevice, s), "hw_learned_init_gradients");
    float l = 0.0f;
    if (!rc) rc = Cuda(cudaMemcpyAsync(&l, h->loss, 4, cudaMemcpyDeviceToHost, s), "hw_learned_init_gradients");
    if (!rc) rc = Cuda(cudaStreamSynchronize(s), "hw_learned_init_gradients");
    if (!rc && loss) *loss = l;
    return rc;
}

// One AdamW step (betas 0.9 / 0.999, eps 1e-8; weight decay on the weight
// matrices only) on the gradients of n rows.
int hw_learned_init_train_step(hw_learned_init* h, const float* d_features, const float* d_targets,
                               const int32_t* d_index, uint32_t n, float lr, float weight_decay, float* loss,
                               void* stream)
{
    int rc = hw_learned_init_gradients(h, d_features, d_targets, d_index, n, nullptr, loss, stream);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    h->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)h->step), c2 = 1.0f - std::pow(b2, (float)h->step);
    struct Seg { size_t off, count; float wd; };
    const Seg segs[] = {{kOffW1, (size_t)kHidden * kFeat, weight_decay}, {kOffB1, kHidden, 0.0f},
                        {kOffW2, (size_t)kHidden * kHidden, weight_decay}, {kOffB2, kHidden, 0.0f},
                        {kOffW3, (size_t)kOut * kHidden, weight_decay}, {kOffB3, kOut, 0.0f}};
    for (const Seg& g : segs)
        AdamWKernel<<<Blocks((long)g.count), 256, 0, s>>>(h->master + g.off, h->grad + g.off, h->m + g.off,
                                                          h->v + g.off, (int)g.count, lr, b1, b2, 1e-8f, g.wd, c1, c2,
                                                          h->wb + g.off);
    return Cuda(cudaGetLastError(), "hw_learned_init_train_step");
}

}   // extern "C"
