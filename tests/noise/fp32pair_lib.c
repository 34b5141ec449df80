/* TEST INFRASTRUCTURE ONLY: fp32pair.h as a shared library for ctypes
 * (tests/test_noise_tolerance.py): forces on slots [0, nact) from all n. */
#include "fp32pair.h"

void fp32pair_force(int order, int n, const double *pred, int nact, double eps2, int split,
                    double *force)
{
    const int F = 3 * (order / 2);
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < nact; ++i)
        fp32pair_force_one(order, n, pred, i, (float)eps2, split, force + (size_t)i * F);
}
