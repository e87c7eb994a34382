// z-line relaxation entry points shared by the C ABI, the momentum predictor,
// the scalar sweeps and the multigrid smoother.
#pragma once

#include "gb_common.cuh"

namespace gb {

//! Scratch slots of a context (each call family owns its slots).
enum ScratchSlot : int {
    kSlotLineNext = 0,
    kSlotLineC,
    kSlotLineE,
    kSlotLineInv,  // 1/m of the factored sweeps
    kSlotLineCp,   // c' of the factored sweeps
    kSlotFirstFree,
    kSlotMultiBase = 24,  // 3 slots (next, 1/m, c') per system of zline_sweeps_multi
    kSlotBatchBase = 48   // zline_sweeps_batch: its systems' fields, then its descriptors
};

enum class LineScratch { automatic, pipelined, shared, global, factored, segmented };

//! `sweeps` z-line Jacobi sweeps into delta (which must hold 0 on entry,
//! ghosts included). change_word (device, may be null) receives the bit
//! pattern of max |change over the last sweep|. No host synchronisation.
template <typename T>
gb_status zline_sweeps(gb_ctx* ctx, const gb_grid& g, int loc, const T* A, const T* ap, const T* rhs, int sweeps,
                       T* delta, unsigned long long* change_word, LineScratch scratch_kind);

//! zline_sweeps for n <= 3 independent systems (each at its own location,
//! each into its own delta, 0 on entry) in one launch per sweep (the
//! factored kernel; more columns in flight than one system gives).
template <typename T>
gb_status zline_sweeps_multi(gb_ctx* ctx, const gb_grid& g, int n, const int* locs, const T* const* A,
                             const T* const* ap, const T* const* rhs, int sweeps, T* const* delta,
                             unsigned long long* const* change_words);

//! zline_sweeps for n systems of different grids (each at its own location,
//! each into its own delta, which this sets to 0) by the segmented sweep over
//! one column work-list: one launch per sweep for each number of warps a
//! block the systems' columns need. change (host, n entries, may be null)
//! receives each system's max |change over the last sweep|, after a wait for
//! the stream; with change null nothing waits.
template <typename T>
gb_status zline_sweeps_batch(gb_ctx* ctx, int n, const gb_grid* grids, const int* locs, const T* const* A,
                             const T* const* ap, const T* const* rhs, int sweeps, T* const* delta, double* change);

//! The line LU-SGS passes (gb_zline_lusgs) into delta (0 on entry, ghosts
//! included); change_word as for zline_sweeps. FP64.
gb_status zline_lusgs(gb_ctx* ctx, const gb_grid& g, int loc, const double* A, const double* ap, const double* rhs,
                      int sweeps, int alternate, double* delta, unsigned long long* change_word);

//! OverrideSync of a field at loc: the high copy of a periodic seam takes the
//! low copy's value.
template <typename T>
void seam_sync(gb_ctx* ctx, const gb_grid& g, int loc, T* f);

}  // namespace gb
