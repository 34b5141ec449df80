// Force-included when compiling the reference's Kepler-era CUDA sources for
// sm_100a: the pre-Volta __shfl_xor (used by SRC/cuda-common.hu:2-3) maps to
// the full-warp __shfl_xor_sync.
#pragma once
#define __shfl_xor(v, m) __shfl_xor_sync(0xffffffffu, (v), (m))
