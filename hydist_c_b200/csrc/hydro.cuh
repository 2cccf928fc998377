// hydro.cuh -- launchers of the hydraulic and sediment kernels.
//
// The simulated time is read by the kernels from State::clock (advanced on
// the device at the start of each half-step), so one step's launches are
// the same every step and can be captured once into a CUDA graph.
#pragma once
#include "common.cuh"

namespace hyd {

// set-up sequence (Onetime_init, segment tables, Htuongdoi, preprocess_data)
void launch_init(const State& S, const Coef& c, cudaStream_t st);
// preprocess_data alone (support_funcs.cpp:482-601): the boundary discharge
// weights hi and the FS boundary scale hmax from the depths
void launch_preprocess(const State& S, const Coef& c, cudaStream_t st);
// Update_Boundary_Value (support_funcs.cpp:603-728) at the device clock's time
void launch_boundary(const State& S, cudaStream_t st);
// segment tables only (from khouot)
void launch_scan_segments(const State& S, cudaStream_t st);
// segment tables + boundary concentration interpolation
void launch_find_limits(const State& S, const Coef& c, cudaStream_t st, Trace* tr);
// hydraulic half-step A: t += dT/2, boundary, x sweep, explicit v, commit
void launch_half_x(const State& S, const Coef& c, cudaStream_t st, Trace* tr);
// hydraulic half-step B: t += dT/2, boundary, y sweep, explicit u, wet/dry,
// commit
void launch_half_y(const State& S, const Coef& c, cudaStream_t st, Trace* tr);
// partitioned hydraulic line sweep: dir 0 = x (columns), 1 = y (rows)
void launch_sweep(const State& S, const Coef& c, int dir, cudaStream_t st);
// partitioned concentration line sweep: dir 0 = i-sweep (columns), 1 = rows;
// the erosion source is on from s_start
void launch_fs_sweep(const State& S, const Coef& c, int dir, double s_start, cudaStream_t st);
// concentration step: xdir = the i-sweep after half-step A; bed: the bed
// change after the j-sweep
void launch_sediment(const State& S, const Coef& c, double s_start, bool xdir, bool bed,
                     cudaStream_t st, Trace* tr);

}  // namespace hyd
