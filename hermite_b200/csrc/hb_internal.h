// hb_internal.h -- host-side declarations shared by the library's units.
#pragma once
#include <cuda_runtime.h>

namespace hb {

struct ForceArgs {
    const void *pred;      // predicted slots, AoSoA32 (FP64 or mixed layout)
    int nchunk;            // number of 32-slot j chunks (padded slots / 32)
    int nact;              // i-particles: slots [0, nact)
    double eps2;
    double *force;         // [nact][F]
    double *partial;       // [S][gridDim.x*TI][F]  (only when S > 1)
    unsigned *counter;     // [gridDim.x], zero between launches
    int *err;              // mapped host flag
};

// One compiled launch shape of the force kernel.
struct ForceVariant {
    int nw;        // warps per CTA
    int ni;        // i-chunks (32 i each) per warp
    int wj;        // warps of an i-group that split the j tile
    int tch;       // 32-slot chunks per j tile
    int ti;        // i per CTA
    int smem;      // dynamic shared memory bytes
    void (*kern)(ForceArgs);
};

int force_variant_count(int order, bool mixed);
const ForceVariant *force_variant(int order, bool mixed, int v);

cudaError_t launch_predict(int order, bool mixed, const double *jp, int n, int npad,
                           double tsys, void *pred, int *err, cudaStream_t s);
cudaError_t launch_potential(int order, const double *jp, int n, int npad, double eps2,
                             double *posm, double *pot, int *err, cudaStream_t s);
cudaError_t run_fma_peak(int mode, int nsm, double *gflops);

}  // namespace hb
