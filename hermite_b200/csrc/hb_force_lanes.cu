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
// sums meet in a fixed xor-shuffle tree.  Each warp predicts its own chunks
// from the raw records (one lane per slot) into shared memory, so a launch
// reads every j record once, and the warps of a CTA take the chunks of its
// j-slice in turn.  The CTAs of the grid are j-slices; the last one to finish
// adds the slices' partials, spread over its threads.  Every sum has a fixed
// association for a given (nact, N), so results are deterministic.
//
// The same job as the reference's force_kernel with its j-blocks
// (SRC/hermite4-titan.cu:189-238, SRC/hermite6-titan.cu:245-299,
// SRC/hermite8-titan.cu:304-364) for the small blocks of the block-step
// scheme; the pair algebra is interact64 (hb_math.cuh).
#include <algorithm>

#include "hb_force.cuh"

namespace hb {
namespace {

constexpr int kLanesWarps = 8;

// Predicts the 32 slots of chunk `chunk` (one per lane) into the predicted
// FP64 chunk layout at dst.  Out of line: the i-particles come from the same
// code, so a particle's i- and j-states are bit-identical and its self term
// is exactly zero.
template <int ORDER>
__device__ __noinline__ void predict_chunk_warp(const double *jp, int chunk, int nbody,
                                                double tsys, double *dst)
{
    constexpr int R = Rec<ORDER>::words;
    const int lane = threadIdx.x & 31, slot = chunk * 32 + lane;
    double x[3], v[3], ac[3] = {0.0, 0.0, 0.0}, jk[3] = {0.0, 0.0, 0.0}, m;
    if (slot < nbody) {
        const double *r = jp + (size_t)slot * R;
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
    constexpr int G = 1 << LOG2G;
    constexpr int F = Frc<ORDER>::words, NC = Pred64<ORDER>::ncomp;
    // per warp: one predicted chunk; after the j loop the same space holds
    // the warps' group sums, then the cross-slice group sums
    constexpr int kWords = kLanesWarps * NC * 32;
    static_assert(kWords >= kLanesWarps * kLanesMaxAct * F, "reduction space");
    static_assert(kWords >= 2 * kLanesWarps * 32 && kWords >= kLanesMaxAct * F, "slice sums");
    __shared__ double sm[kWords];
    __shared__ unsigned s_last;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int p = lane >> LOG2G, g = lane & (G - 1);
    const int S = gridDim.x, sl = blockIdx.x, nact = a.nact;
    double *my = sm + w * NC * 32;

    // i-particle p (lanes of groups p >= nact compute a copy of the last one
    // and are dropped at the end); the i-particles are slots 0..nact-1 of chunk 0
    predict_chunk_warp<ORDER>(a.jp, 0, a.nbody, a.tsys, my);
    __syncwarp();
    Body64 I;
    load_i64<ORDER>(my, 0, min(p, nact - 1), I);
    __syncwarp();

    double f[F];
#pragma unroll
    for (int q = 0; q < F; ++q) f[q] = 0.0;
    const int c0 = (int)((long long)sl * a.nchunk / S);
    const int c1 = (int)((long long)(sl + 1) * a.nchunk / S);
    for (int c = c0 + w; c < c1; c += kLanesWarps) {
        predict_chunk_warp<ORDER>(a.jp, c, a.nbody, a.tsys, my);
        __syncwarp();
        chunk64_lanes<ORDER, LOG2G>(my, I, a.eps2, f);
        __syncwarp();
    }
    // the G lanes of a group: a fixed butterfly
#pragma unroll
    for (int o = G >> 1; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < F; ++q) f[q] += __shfl_xor_sync(0xffffffffu, f[q], o);
    __syncthreads();                     // every warp is done with its chunk
    double *red = sm;                    // [warp][i][F]
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
    double *grp = sm;
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

cudaError_t launch_force_lanes(int order, const ForceArgs &a, int nsm, cudaStream_t s)
{
    if (a.nact < 1 || a.nact > kLanesMaxAct || a.nchunk < 1) return cudaErrorInvalidValue;
    const int log2g = lanes_log2g(a.nact);                // P = 2^(5 - log2g) >= nact
    // j-slices of at least two chunks a warp, at most two CTAs per SM
    const int S = std::max(1, std::min(2 * nsm, a.nchunk / (2 * kLanesWarps)));
    const dim3 grid(S), block(kLanesWarps * 32);
    // groups of G = 2..32 lanes (nact <= 16 leaves at least two lanes per i)
    static_assert(kLanesMaxAct <= 16, "one lane per i-particle is the tiled kernel's job");
    using K = void (*)(ForceArgs);
    static const K table[3][5] = {
        {force_lanes_kernel<4, 1>, force_lanes_kernel<4, 2>, force_lanes_kernel<4, 3>,
         force_lanes_kernel<4, 4>, force_lanes_kernel<4, 5>},
        {force_lanes_kernel<6, 1>, force_lanes_kernel<6, 2>, force_lanes_kernel<6, 3>,
         force_lanes_kernel<6, 4>, force_lanes_kernel<6, 5>},
        {force_lanes_kernel<8, 1>, force_lanes_kernel<8, 2>, force_lanes_kernel<8, 3>,
         force_lanes_kernel<8, 4>, force_lanes_kernel<8, 5>}};
    const int oi = order == 4 ? 0 : order == 6 ? 1 : order == 8 ? 2 : -1;
    if (oi < 0) return cudaErrorInvalidValue;
    table[oi][log2g - 1]<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace hb
