/*
 * hydist_uvz_compat.h -- the reference's UVZSolver kernels with their C++
 * signatures (UVZSolver_multithread.h:6-55), for CUDA programs that drive
 * the ADI half-steps themselves, as the reference's engine.cpp does. Link
 * with libhydist_b200.so in place of UVZSolver_multithread.cpp and
 * gtsv.cpp; the reference's support_funcs.cpp and sediment_transport.cpp
 * stay the caller's.
 *
 * Every kernel keeps the reference's launch contract (which cell or line a
 * thread takes from its launch shape and the index arguments) and writes
 * the intermediate arrays of Array_Pointers in the reference's layout, so
 * the caller's own kernels between them read them unchanged:
 *   f1..f5, a2, c2, d2 (preindex) and a1..d1 (abcd): line * (N+2) + i for
 *     the x sweep (line = column j), line * (M+2) + j for the y sweep;
 *   AA, BB, CC, DD (matrix_coeff) and x (tridiagSolver): line * (2N+1) or
 *     line * (2M+1) + row, a segment's system from row 2*first;
 *   SN: line * 20 + segment, the index of the system's last row.
 * Sizes the caller allocates: (N+3)*(M+3) doubles for each of f1..f5,
 * a1..d1, a2, c2, d2; 2*(N+3)*(M+3) for each of AA..DD, x, Ap, Bp, ep;
 * 20*(max(M,N)+1) ints for SN, which the y sweep writes for rows up to N.
 * The reference's supporting_arrays_alloc (loader.cpp:333-362) allocates
 * less (M*N+2*max(M,N), 2*M*N+4*max(M,N) and 20*max(M,N)), which the
 * reference's own kernels overrun on meshes whose last row or column is
 * wet.
 *
 * Link the program with the shared CUDA runtime (nvcc -cudart shared): a
 * launch from the program hands its configuration to the kernel's stub in
 * this library through the runtime, and a static runtime copy in the
 * program is not the library's.
 *
 * These kernels are the kernel-level drop-in, not the fast path:
 * Hydraulic_Calculation (hydist_compat.h) and hydist_step run a half-step
 * without the intermediate arrays, in a few fused kernels.
 *
 * A translation unit must not include both this header and the reference's
 * UVZSolver_multithread.h.
 */
#ifndef HYDIST_UVZ_COMPAT_H
#define HYDIST_UVZ_COMPAT_H

#include "hydist_compat.h"

/* y sweep (VZ): rows i = startidx..endidx, columns 2..M */
__global__ void VZSolver_calculate_preindex(int startidx, int endidx, Argument_Pointers* arg,
                                            Array_Pointers* arr, Constant_Coeffs* coeffs);
__global__ void VZSolver_calculate_abcd(int startidx, int endidx, Argument_Pointers* arg,
                                        Array_Pointers* arr, Constant_Coeffs* coeffs);
__global__ void VZSolver_calculate_matrix_coeff(int startidx, int endidx, double NANGDAY,
                                                Argument_Pointers* arg, Array_Pointers* arr);
/* as the reference: the column is tested against endidx (columns <= endidx) */
__global__ void VZSolver_extract_solution(int startidx, int endidx, double NANGDAY,
                                          Argument_Pointers* arg, Array_Pointers* arr);
/* explicit v on rows startidx..endidx (t is not used, as in the reference) */
__global__ void solveV(double t, int startidx, int endidx, Argument_Pointers* arg,
                       Constant_Coeffs* coeffs);
/* segment-end v of rows blockIdx.y*blockDim.y+threadIdx.y+startidx */
__global__ void update_margin_elem_V(int startidx, int endidx, double NANGDAY,
                                     Argument_Pointers* arg);

/* x sweep (UZ): columns j = startidx..endidx, rows 2..N */
__global__ void UZSolver_extract_solution(int startidx, int endidx, double NANGDAY,
                                          Argument_Pointers* arg, Array_Pointers* arr);
__global__ void UZSolver_calculate_preindex(int startidx, int endidx, Argument_Pointers* arg,
                                            Array_Pointers* arr, Constant_Coeffs* coeffs);
__global__ void UZSolver_calculate_abcd(int startidx, int endidx, Argument_Pointers* arg,
                                        Array_Pointers* arr, Constant_Coeffs* coeffs);
__global__ void UZSolver_calculate_matrix_coeff(int startidx, int endidx, double NANGDAY,
                                                Argument_Pointers* arg, Array_Pointers* arr);
/* explicit u on rows 1..N, columns startidx..endidx */
__global__ void solveU(double t, int startidx, int endidx, Argument_Pointers* arg,
                       Constant_Coeffs* coeffs);
/* segment-end u of columns blockIdx.y*blockDim.y+threadIdx.y+startidx */
__global__ void update_margin_elem_U(int startidx, int endidx, double NANGDAY,
                                     Argument_Pointers* arg);

/* the segments of line blockIdx.y+startidx (isU: columns, else rows),
 * segment s's system at line*tridiag_coeff_width + first*jumpstep +
 * jumpstep%2 with SN[line*20+s]+1 rows; Ap, Bp, ep are its scratch. Also
 * used by the reference's concentration sweeps (jumpstep 1). */
__global__ void tridiagSolver(bool print, bool isU, int startidx, int endidx, int jumpstep,
                              int tridiag_coeff_width, Argument_Pointers* arg, Array_Pointers* arr);
/* the segments of line threadIdx.x+startidx through
 * gtsv_spike_partial_diag_pivot_v1 (hydist_gtsv_device.cuh), m = SN as the
 * reference passes it */
__global__ void tridiagSolver_v2(bool print, bool isU, int startidx, int endidx, int jumpstep,
                                 int tridiag_coeff_width, Argument_Pointers* arg,
                                 Array_Pointers* arr);

#endif
