// cufsp_march.h -- launch arguments of the TMA-fed marching KRONECKER kernel (cufsp_kron_march.cu).
#pragma once
#include <cuda_runtime.h>

#include "cufsp_internal.h"

namespace cufsp {

constexpr int kMarchMaxSlots = 6;
constexpr int kMarchMaxR = 8;  // tile rows (bounded: the y pipeline keeps one register set per row)

struct MarchArgs {
    const double2 *__restrict__ gtab;   // [Q][NR] outer factor products (shifted, unshifted)
    const double *__restrict__ tables;  // [NR][tab_stride]
    const int *__restrict__ nu;         // [NR][ns]
    const double *__restrict__ d_alpha; // nullable
    const int *__restrict__ d_skip;     // nullable
    int *err;                           // watchdog flag (device)
    int n, P, L, RP, Z;                 // states, plane size, row length, rows per plane, planes
    int ns, k, tab_stride;
    int R;                              // tile rows
    int hr_lo, hr_hi;                   // halo rows below / above the tile
    int hz_lo, hz_hi;                   // a step at plane z reads planes z - hz_lo .. z + hz_hi
    int slots;                          // ring size (hz_lo + hz_hi + 2)
    int slot_elems;                     // doubles per slot (guards + staged rows), even
    int guard;                          // guard doubles before the first staged row, even
    int row_tiles, zseg;                // grid = row_tiles x ceil(Z / zseg)
    int dims[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
    int dz[CUFSP_MAX_REACTIONS];        // nu_{r,z}: source plane z - dz
    int soff[CUFSP_MAX_REACTIONS];      // in-slot offset of the source: (hr_lo - drow_r) * L - dp_r
    double coef[CUFSP_MAX_REACTIONS];
};

using MarchKernel = void (*)(const MarchArgs, const double *, double *);
MarchKernel pick_march_kernel(int NR, int V, bool accum);

}  // namespace cufsp
