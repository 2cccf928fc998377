// hydro.cuh -- launchers of the hydraulic and sediment kernels.
//
// The simulated time is read by the kernels from State::clock (advanced on
// the device at the start of each half-step), so one step's launches are
// the same every step and can be captured once into a CUDA graph.
#pragma once
#include "common.cuh"

namespace hyd {

// Every launcher exists for R = double (the plain form) and R = float (the
// FP32 form), instantiated where it is defined.

// set-up sequence (Onetime_init, segment tables, Htuongdoi, preprocess_data)
template <class R>
void launch_init(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st);
// preprocess_data alone (support_funcs.cpp:482-601): the boundary discharge
// weights hi and the FS boundary scale hmax from the depths
template <class R>
void launch_preprocess(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st);
// Update_Boundary_Value (support_funcs.cpp:603-728) at the device clock's time
template <class R>
void launch_boundary(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st);
// segment tables only (from khouot; dry: with the drying pass of
// Reset_states_vertical applied to the mask first)
template <class R>
void launch_scan_segments(const StateT<R>& S, const CoefT<R>& c, bool dry, cudaStream_t st,
                          const Batch<R>& b = {});
// segment tables + boundary concentration interpolation
template <class R>
void launch_find_limits(const StateT<R>& S, const CoefT<R>& c, bool dry, cudaStream_t st,
                        Trace* tr, const Batch<R>& b = {});
// hydraulic half-step A: t += dT/2, boundary, x sweep, explicit v, commit;
// sed: a concentration step follows (the commit computes its speeds and
// diffusivities, Find_VTH + hesoK). With a batch (b.n > 0) every launch
// covers all of its members; S and c are then those of one member (the
// sizes and the options that shape the launches, the same for all).
template <class R>
void launch_half_x(const StateT<R>& S, const CoefT<R>& c, bool sed, cudaStream_t st, Trace* tr,
                   const Batch<R>& b = {});
// hydraulic half-step B: t += dT/2, boundary, y sweep, explicit u, wet/dry,
// commit; sed as above; qb: the bed change follows the step's concentration
// j-sweep (the commit computes its flux, Calculate_Qb)
template <class R>
void launch_half_y(const StateT<R>& S, const CoefT<R>& c, bool sed, cudaStream_t st, Trace* tr,
                   const Batch<R>& b = {}, bool qb = false);
// partitioned hydraulic line sweep: dir 0 = x (columns), 1 = y (rows)
template <class R>
int launch_sweep(const StateT<R>& S, const CoefT<R>& c, int dir, cudaStream_t st,
                 const Batch<R>& b = {});
// partitioned concentration line sweep: dir 0 = i-sweep (columns), 1 = rows;
// the erosion source is on from StateT::src_start
template <class R>
int launch_fs_sweep(const StateT<R>& S, const CoefT<R>& c, int dir, cudaStream_t st,
                    const Batch<R>& b = {});
// concentration step (after a half-step launched with sed): xdir = the
// i-sweep after half-step A; bed: the bed change after the j-sweep
template <class R>
void launch_sediment(const StateT<R>& S, const CoefT<R>& c, bool xdir, bool bed, cudaStream_t st,
                     Trace* tr, const Batch<R>& b = {});

// the bed change fed back into h, htaiz, Kx1, Ky1 (HydistOptions::bed_feedback)
template <class R>
void launch_bed_feedback(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st,
                         const Batch<R>& b = {});

}  // namespace hyd
