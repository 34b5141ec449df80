// hb_force_lanes.cu -- FP64 force on a handful of active particles.
//
// The tiled force kernel (hb_force.cuh) gives every lane of a warp its own
// i-particle, so a block step with nact < 32 active particles leaves
// 32 - nact lanes idle: at nact = 1 the j sum runs at 1/32 of the FP64 pipe
// (about 24 us of arithmetic at N = 262144, 6th order, where the j records
// take 6.5 us to stream from HBM).
//
// Here a warp's 32 lanes form P groups of G = 32/P lanes, P = nact rounded
// up to a power of two (nact <= 16, so G >= 2; from 17 on, one lane per i,
// the tiled kernel measured faster at N >= 2^18).  The G lanes of group p share
// i-particle p and take every G-th j of each 32-slot chunk; their partial
// sums meet in a fixed xor-shuffle tree.  The warps of a CTA take the chunks
// of its j-slice in turn; each warp brings its chunks' raw records into shared
// memory by bulk copies, two in flight (every wait bounded), and predicts them
// there (one lane per slot), so a launch reads every j record once.  The CTAs of the grid are j-slices; the last one to finish
// adds the slices' partials, spread over its threads.  Every sum has a fixed
// association for a given (nact, N), so results are deterministic.
//
// The same job as the reference's force_kernel with its j-blocks
// (SRC/hermite4-titan.cu:189-238, SRC/hermite6-titan.cu:245-299,
// SRC/hermite8-titan.cu:304-364) for the small blocks of the block-step
// scheme; the pair algebra is interact64 (hb_math.cuh).
#include <algorithm>
#include <mutex>

#include "hb_force.cuh"

namespace hb {
namespace {

constexpr int kLanesWarps = 8;
constexpr int kLanesStages = 2;     // raw chunks in flight per warp

// Dynamic shared memory of one CTA: per warp, kLanesStages raw chunks (32
// records each, AoS, filled by bulk copies) and one predicted chunk; then
// the warps' mbarriers.  After the j loop the front of it holds the warps'
// group sums and then the cross-slice group sums.
template <int ORDER>
struct LanesSmem {
    static constexpr int raw = 32 * Rec<ORDER>::bytes;        // 3584 / 5120 / 6656
    static constexpr int pred = Pred64<ORDER>::ncomp * 32 * 8;
    static constexpr int warp = kLanesStages * raw + pred;
    static constexpr int bar_off = kLanesWarps * warp;
    static constexpr int bytes = bar_off + kLanesWarps * kLanesStages * 8;
    static_assert(raw % 16 == 0 && pred % 16 == 0, "bulk copies need 16-byte offsets");
    static_assert(bar_off >= kLanesWarps * kLanesMaxAct * Frc<ORDER>::words * 8, "reduction space");
    static_assert(bar_off >= 2 * kLanesWarps * 32 * 8, "slice sums");
};

// Predicts the 32 slots of chunk `chunk` (one per lane) from their raw
// records in shared memory into the predicted FP64 chunk layout at dst.  Out
// of line: the i-particles come from the same code, so a particle's i- and
// j-states are bit-identical and its self term is exactly zero.
template <int ORDER>
__device__ __noinline__ void predict_raw_chunk(const double *raw, int chunk, int nbody,
                                               double tsys, double *dst)
{
    constexpr int R = Rec<ORDER>::words;
    const int lane = threadIdx.x & 31, slot = chunk * 32 + lane;
    double x[3], v[3], ac[3] = {0.0, 0.0, 0.0}, jk[3] = {0.0, 0.0, 0.0}, m;
    if (slot < nbody) {
        const double *r = raw + lane * R;
        predict_slot<ORDER>(r, tsys, x, v, ac, jk);
        m = r[3];
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) { x[k] = pad_position(slot, k); v[k] = 0.0; }
        m = 0.0;
    }
    double *c = dst + lane;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        c[(P64_X + k) * 32] = x[k];
        c[(P64_V + k) * 32] = v[k];
        if constexpr (ORDER >= 6) c[(P64_A + k) * 32] = ac[k];
        if constexpr (ORDER >= 8) c[(P64_J + k) * 32] = jk[k];
    }
    c[P64_M * 32] = m;
}

template <int ORDER, int LOG2G>
__global__ void __launch_bounds__(kLanesWarps * 32)
force_lanes_kernel(ForceArgs a)
{
    using L = LanesSmem<ORDER>;
    constexpr int G = 1 << LOG2G, STG = kLanesStages;
    constexpr int F = Frc<ORDER>::words, R = Rec<ORDER>::words;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned s_last;
    __shared__ int s_fail;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int p = lane >> LOG2G, g = lane & (G - 1);
    const int S = gridDim.x, sl = blockIdx.x, nact = a.nact;
    unsigned char *wraw = smem + w * L::warp;                            // this warp's raw stages
    double *my = reinterpret_cast<double *>(wraw + STG * L::raw);        // its predicted chunk
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::bar_off) + w * STG;

    if (tid == 0) s_fail = 0;
    if (lane == 0) {
#pragma unroll
        for (int st = 0; st < STG; ++st) mbar_init(&bar[st], 1);
        fence_mbar_init();
    }
    __syncthreads();

    // This warp's loads: chunk 0 (the i-particles are its first nact slots),
    // then chunks c0 + w, c0 + w + kLanesWarps, ... of the CTA's j-slice.
    const int c0 = (int)((long long)sl * a.nchunk / S);
    const int c1 = (int)((long long)(sl + 1) * a.nchunk / S);
    const int nload = 1 + (c0 + w < c1 ? (c1 - c0 - w + kLanesWarps - 1) / kLanesWarps : 0);
    auto chunk_of = [&](int q) { return q == 0 ? 0 : c0 + w + (q - 1) * kLanesWarps; };
    auto issue = [&](int q) {   // lane 0 only
        const int st = q % STG;
        mbar_arrive_expect_tx(&bar[st], (uint32_t)L::raw);
        bulk_load(wraw + st * L::raw, a.jp + (size_t)chunk_of(q) * 32 * R, (uint32_t)L::raw, &bar[st]);
    };
    if (lane == 0)
        for (int q = 0; q < STG && q < nload; ++q) issue(q);

    Body64 I;
    double f[F];
#pragma unroll
    for (int q = 0; q < F; ++q) f[q] = 0.0;
    int failed_at = -1;
    for (int q = 0; q < nload; ++q) {
        const int st = q % STG;
        const bool got = mbar_wait_bounded(&bar[st], (uint32_t)((q / STG) & 1), a.spin);
        if (!__all_sync(0xffffffffu, got)) { failed_at = q; break; }
        predict_raw_chunk<ORDER>(reinterpret_cast<const double *>(wraw + st * L::raw), chunk_of(q),
                                 a.nbody, a.tsys, my);
        __syncwarp();                    // the raw stage is read: refill it
        if (lane == 0 && q + STG < nload) issue(q + STG);
        if (q == 0)
            load_i64<ORDER>(my, 0, min(p, nact - 1), I);   // lanes of groups p >= nact: a copy
        else
            chunk64_lanes<ORDER, LOG2G>(my, I, a.eps2, f);
        __syncwarp();                    // `my` is read: the next prediction may overwrite it
    }
    if (failed_at >= 0) {
        // leave no bulk copy writing into shared memory after this CTA ends
        if (lane == 0) {
            for (int q = failed_at; q < nload && q < failed_at + STG; ++q)
                mbar_wait_bounded(&bar[q % STG], (uint32_t)((q / STG) & 1));
            atomicOr(&s_fail, 1);
        }
    }
    __syncthreads();
    if (s_fail) {
        if (tid == 0) raise_error(a.err, kErrWaitTimeout);
        return;
    }
    // the G lanes of a group: a fixed butterfly
#pragma unroll
    for (int o = G >> 1; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < F; ++q) f[q] += __shfl_xor_sync(0xffffffffu, f[q], o);
    double *red = reinterpret_cast<double *>(smem);          // [warp][i][F]
    if (g == 0 && p < nact)
#pragma unroll
        for (int q = 0; q < F; ++q) red[(w * kLanesMaxAct + p) * F + q] = f[q];
    __syncthreads();

    const int V = nact * F;
    for (int e = tid; e < V; e += blockDim.x) {
        double v = red[e];
#pragma unroll
        for (int ww = 1; ww < kLanesWarps; ++ww) v += red[ww * kLanesMaxAct * F + e];
        if (S == 1) a.force[e] = v;
        else a.partial[(size_t)sl * kLanesMaxAct * F + e] = v;
    }
    if (S == 1) return;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(&a.counter[0], 1u) == (unsigned)(S - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the slices' sum, spread over the CTA: thread t = k*V + e adds slices
    // k, k+K, ... of value e into 8 interleaved sums (8 loads in flight),
    // combined pairwise; then each value's K group sums in group order
    const int K = max(1, (int)blockDim.x / V);
    double *grp = reinterpret_cast<double *>(smem);
    for (int t = tid; t < K * V; t += blockDim.x) {
        const int k = t / V, e = t - k * V;
        double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int s2 = k;
        for (; s2 + 7 * K < S; s2 += 8 * K)
#pragma unroll
            for (int u = 0; u < 8; ++u)
                acc[u] += __ldcg(a.partial + (size_t)(s2 + u * K) * kLanesMaxAct * F + e);
#pragma unroll
        for (int u = 0; u < 7; ++u)
            if (s2 + u * K < S) acc[u] += __ldcg(a.partial + (size_t)(s2 + u * K) * kLanesMaxAct * F + e);
        grp[t] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    }
    __syncthreads();
    for (int e = tid; e < V; e += blockDim.x) {
        double v = grp[e];
        for (int k = 1; k < K; ++k) v += grp[k * V + e];
        a.force[e] = v;
    }
    if (tid == 0) a.counter[0] = 0u;
}

}  // namespace

namespace {

using LanesKernel = void (*)(ForceArgs);
const LanesKernel kLanesTable[3][5] = {   // groups of G = 2..32 lanes
    {force_lanes_kernel<4, 1>, force_lanes_kernel<4, 2>, force_lanes_kernel<4, 3>,
     force_lanes_kernel<4, 4>, force_lanes_kernel<4, 5>},
    {force_lanes_kernel<6, 1>, force_lanes_kernel<6, 2>, force_lanes_kernel<6, 3>,
     force_lanes_kernel<6, 4>, force_lanes_kernel<6, 5>},
    {force_lanes_kernel<8, 1>, force_lanes_kernel<8, 2>, force_lanes_kernel<8, 3>,
     force_lanes_kernel<8, 4>, force_lanes_kernel<8, 5>}};
constexpr int kLanesBytes[3] = {LanesSmem<4>::bytes, LanesSmem<6>::bytes, LanesSmem<8>::bytes};

// Per device (up to 64): the kernels' shared-memory attribute set once, and
// the resident CTAs per SM of each order.
std::mutex g_lanes_mu;
unsigned long long g_lanes_ready = 0;
int g_lanes_per_sm[64][3];

cudaError_t lanes_setup(int oi, int *per_sm)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_lanes_mu);
    if (!(g_lanes_ready >> dev & 1ull)) {
        for (int o = 0; o < 3; ++o) {
            for (int v = 0; v < 5; ++v) {
                e = cudaFuncSetAttribute(kLanesTable[o][v], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kLanesBytes[o]);
                if (e != cudaSuccess) return e;
            }
            int nb = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kLanesTable[o][4], kLanesWarps * 32,
                                                              kLanesBytes[o]);
            if (e != cudaSuccess) return e;
            g_lanes_per_sm[dev][o] = std::max(1, nb);
        }
        g_lanes_ready |= 1ull << dev;
    }
    *per_sm = g_lanes_per_sm[dev][oi];
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_force_lanes(int order, const ForceArgs &a, int nsm, cudaStream_t s)
{
    static_assert(kLanesMaxAct <= 16, "one lane per i-particle is the tiled kernel's job");
    if (a.nact < 1 || a.nact > kLanesMaxAct || a.nchunk < 1) return cudaErrorInvalidValue;
    const int oi = order == 4 ? 0 : order == 6 ? 1 : order == 8 ? 2 : -1;
    if (oi < 0) return cudaErrorInvalidValue;
    int per_sm = 1;
    cudaError_t e = lanes_setup(oi, &per_sm);
    if (e != cudaSuccess) return e;
    const int log2g = lanes_log2g(a.nact);                // P = 2^(5 - log2g) >= nact, G >= 2
    // j-slices of at least two chunks a warp, all CTAs resident at once
    const int S = std::max(1, std::min(std::min(2, per_sm) * nsm, a.nchunk / (2 * kLanesWarps)));
    kLanesTable[oi][log2g - 1]<<<S, kLanesWarps * 32, kLanesBytes[oi], s>>>(a);
    return cudaGetLastError();
}

}  // namespace hb
