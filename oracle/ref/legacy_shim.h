/* legacy_shim.h -- forced-include shim that lets EZLDA's sources (written for sm_35,
 * before CUDA 9) compile for sm_100a: the pre-Volta warp intrinsics __shfl, __shfl_up,
 * __shfl_down and __ballot no longer exist and map onto their full-warp _sync forms.
 * Every use in the kernels the harness launches sits in warp-uniform control flow
 * (checked by reading EZLDA/utility.cu), so the full mask is exact there.
 * TEST INFRASTRUCTURE: used only to build the reference into oracle/_ref. */
#pragma once
#include <cuda_runtime.h>
#define __shfl(v, l, ...) __shfl_sync(0xffffffffu, (v), (l), ##__VA_ARGS__)
#define __shfl_up(v, d, ...) __shfl_up_sync(0xffffffffu, (v), (d), ##__VA_ARGS__)
#define __shfl_down(v, d, ...) __shfl_down_sync(0xffffffffu, (v), (d), ##__VA_ARGS__)
#define __ballot(p) __ballot_sync(0xffffffffu, (p))
