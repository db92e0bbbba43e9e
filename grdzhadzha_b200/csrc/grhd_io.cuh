// grhd_io.cuh -- diagnostics reduction and checkpoint layout of the
// reference's example drivers, on the device.
//
//  * compute_diagnostics (Examples/GRHDLevelDataKerrSchildDisk/
//    Main_GRHDLevelDataKerrSchildDisk.cpp:223-290, the same in the binary
//    drivers): proper-volume sums of D and tau (all cells, and D over cells
//    denser than 10 x the atmosphere floor) and the maxima of rho, p, |v|
//    and W over the interior;
//  * the KITPCHK1 checkpoint state (Examples/GRHDLevelDataBinaryPNKITPDisk/
//    Main_GRHDLevelDataBinaryPNKITPDisk.cpp:1191-1590): all NUM_VARS
//    components interleaved per cell over the domain grown by the ghosts,
//    value index ((k ny + j) nx + i) NUM_VARS + component, the GRHD
//    components last.
#pragma once

#include "grhd_kernels.cuh"

namespace grhd {

// Per-block partial results of the diagnostics: [block][7] (three sums,
// four maxima); `blocks` is the launch's grid size.
int diagnostics_blocks(const BoxDev &b);
void launch_diagnostics(const double *state, const BoxDev &b,
                        const Background &bg, const Options &o,
                        double *partial, cudaStream_t s);

// SoA state (11 components, stride b.cs, over the ghosted box) to the
// interleaved checkpoint layout with `ncomp` components (the first
// ncomp - 11 written as zero), and back.
void launch_state_to_checkpoint(const double *state, const BoxDev &b,
                                int ncomp, double *out, cudaStream_t s);
void launch_checkpoint_to_state(const double *in, const BoxDev &b, int ncomp,
                                double *state, cudaStream_t s);

// LevelData::exchange between two boxes of a level: the first `ncomp`
// components of the cells [lo, hi] (level index space) from `src` (box sb)
// to `dst` (box db).
void launch_copy_region(double *dst, const BoxDev &db, const double *src,
                        const BoxDev &sb, const int lo[3], const int hi[3],
                        int ncomp, cudaStream_t s);

// The first `ncomp` components of the region [lo, hi] (inside the ghosted
// box) into (pack) or out of a packed buffer [component][k][j][i].
void launch_region(bool pack, double *state, const BoxDev &b, double *buf,
                   const int lo[3], const int hi[3], int ncomp,
                   cudaStream_t s);

} // namespace grhd
