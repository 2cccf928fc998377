// hydro.cuh -- launchers of the hydraulic and sediment kernels.
#pragma once
#include "common.cuh"

namespace hyd {

// set-up sequence (Onetime_init, segment tables, Htuongdoi, preprocess_data)
void launch_init(const State& S, const Coef& c, cudaStream_t st);
// segment tables only (from khouot)
void launch_scan_segments(const State& S, cudaStream_t st);
// segment tables + boundary concentration interpolation
void launch_find_limits(const State& S, const Coef& c, cudaStream_t st, Trace* tr);
// hydraulic half-step A: boundary at t, x sweep, explicit v, commit
void launch_half_x(const State& S, const Coef& c, double t, cudaStream_t st, Trace* tr);
// hydraulic half-step B: boundary at t, y sweep, explicit u, wet/dry, commit
void launch_half_y(const State& S, const Coef& c, double t, cudaStream_t st, Trace* tr);
// concentration sweeps: xdir = the i-sweep after half-step A
void launch_sediment(const State& S, const Coef& c, double t, double s_start, bool xdir,
                     cudaStream_t st, Trace* tr);

}  // namespace hyd
