// ipm_kernels.cuh -- per-iteration vector kernels of the Mehrotra predictor-corrector method.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace sov {

// Scalars of one iteration, written on the device, read by the host once per iteration.
struct IpmScalars {
  // residual phase (interior_point.cpp:572-602, qp_interior_point.cpp:2978-3000)
  double rp_max, rd_max, xs, cx, xqx, qx_max;
  double mu, p_res, d_res, gap, metric;
  // direction phase
  double ratio_p, ratio_d;    // step_to_bound of the last direction (<= 1)
  double alpha_p_aff, alpha_d_aff, mu_aff, sigma;
  double alpha_p, alpha_d;    // step taken
  // solver health
  int fail, drops, err, skipped;
};

struct IpmDev {
  int m, n;
  // A in CSR (rows) and CSC (columns), scaled
  const int* row_ptr;
  const int* col_idx;
  const double* rval;
  const int* col_ptr;
  const int* row_idx;
  const double* cval;
  const double* b;
  const double* c;
  const double* qdiag;      // QP: diagonal of Q (null for LP)
  const uint8_t* free_col;  // QP: 1 = no barrier (null for LP)
  int qp;
  int has_quadratic;
  // QP whose Hessian couples variables: Q over the IPM columns, CSC with both triangles (null and
  // 0 for separable Hessians, which use qdiag alone)
  const int* q_ptr;
  const int* q_idx;
  const double* q_val;
  int q_coupled;
  // 1 while the starting-point system (every column weight 1) is solved: the matrix-free normal
  // operator of the mixed path then uses weight 1 too
  int start_system;
  double comp_count;        // n (LP) or max(1, #bounded) (QP)
  double bnorm, cnorm, objective_offset, tau;
  // iterate and work vectors
  double *x, *y, *s;
  double *dx, *ds, *dxa, *dsa;
  double *rp, *rd;
  double* z;                // Newton right-hand side / solution (padded to the solver's order)
  double* dy;               // dy of the last direction (== z in y-space)
  // x-space QP (every row has a slack, Q_jj > 0 on structural columns): K dx_x = rhs, then dy, dw
  int xspace;
  int nx;                   // structural columns
  const int* slack_of_row;  // m
  const double* sigma;      // m: slack coefficient of the row (+1 / -1)
  double* tr;               // m scratch
  IpmScalars* sc;
  // long rows (wide LPs): a CTA per row in the row kernels, and the Newton right-hand side's
  // column terms computed once per column into coltmp (n) instead of once per entry
  int row_block;
  double* coltmp;
  // a row longer than a piece (a dense row): every row kernel walks the rows as warp-sized pieces
  // (row_pieces in sparse.hpp) and finishes the cut rows in a combine launch
  const int4* row_piece;
  int row_pieces;
  const int4* row_comb;
  int row_combs;
  double* row_partial;
  // grid reduction scratch
  double* partials;         // 8 * max_blocks
  unsigned* counter;
};

enum RhsMode : int { kRhsAffine = 0, kRhsCorrector = 1 };

// rp = b - A x, rd = c + Q x - A'y - s; fills sc->{rp_max, rd_max, xs, cx, mu, p_res, d_res, gap}
void launch_residuals(const IpmDev& d, cudaStream_t st, int* launches);
// z = rp + A tmp (Newton right-hand side of the normal equations)
void launch_newton_rhs(const IpmDev& d, int mode, cudaStream_t st, int* launches);
// dx, ds from dy = z; ratio tests; affine -> alpha_aff, mu_aff, sigma; corrector -> alpha
void launch_direction(const IpmDev& d, int mode, cudaStream_t st, int* launches);
// x, s, y update with the 1e-14 floors
void launch_update(const IpmDev& d, cudaStream_t st, int* launches);
// starting point: z = b - A 1 (rhs of the least-squares push)
void launch_start_rhs(const IpmDev& d, cudaStream_t st, int* launches);
// starting point from dy = z (interior_point.cpp:497-503; qp_interior_point.cpp:2931-2947)
void launch_start_point(const IpmDev& d, cudaStream_t st, int* launches);
// matrix-free normal product out = A diag(w) A' v + reg v, w from the iterate (mixed-precision PCG)
void launch_normal_matvec(const IpmDev& d, const double* v, double* tmp_n, double* out, double reg,
                          cudaStream_t st);

// x-space counterparts (xspace == 1)
void launch_newton_rhs_x(const IpmDev& d, int mode, cudaStream_t st, int* launches);
void launch_direction_x(const IpmDev& d, int mode, cudaStream_t st, int* launches);
void launch_start_rhs_x(const IpmDev& d, cudaStream_t st, int* launches);
void launch_start_dy_x(const IpmDev& d, cudaStream_t st, int* launches);
// K_jj += Q_jj + h_j (mode 1) or += 1 (start, mode 0); same on the recorded diagonal
void launch_xspace_diag(const IpmDev& d, int mode, double* M, int layout_ld, double* diag, cudaStream_t st);

// Coupled-Hessian QP (q_coupled == 1): the Newton system is reduced with H = Q + diag(h) held dense
// and factored (h_j = s_j/x_j, 0 for free columns, 1 at the start), so that
//   M = A H^-1 A' (+ reg on the diagonal) dy = rp - A H^-1 r1,   dx = H^-1 (r1 + A'dy)
// with r1 = -rd + rxs/x (free: -rd) as in the separable path (qp_interior_point.cpp:2832-2844).
// H += diag(h) on a copy of dense Q (column-major, ld); diag[j] = H_jj for the pivot rule
void launch_hessian_diag(const IpmDev& d, bool start, double* H, int ld, double* diag, cudaStream_t st);
// Y[:, i] = row i of A (Y zeroed by the caller, column-major, ld)
void launch_rows_to_columns(const IpmDev& d, double* Y, int ld, cudaStream_t st);
// lower triangle of M = A Y (Y = H^-1 A', ld_y), reg added on the diagonal; diag[i] = M_ii
void launch_form_normal(const IpmDev& d, const double* Y, int ld_y, double* M, int ld_m, double reg, double* diag,
                        cudaStream_t st);
// r1 of the current mode into v (entries n.. untouched)
void launch_hessian_r1(const IpmDev& d, int mode, double* v, cudaStream_t st);
// z = base - A v (v = H^-1 r1; base = rp, or zero when null)
void launch_rows_minus(const IpmDev& d, const double* v, const double* base, cudaStream_t st);
// v = r1 + A'dy (dy = z)
void launch_hessian_w(const IpmDev& d, int mode, double* v, cudaStream_t st);
// dx = dxv (= H^-1 (r1 + A'dy)), ds, ratio tests and step lengths as launch_direction
void launch_direction_dx(const IpmDev& d, int mode, const double* dxv, cudaStream_t st, int* launches);

// Mehrotra's QP start (qp_interior_point.cpp:2891-2928), with dy of the start system in z:
// xt = 1 + A'dy into xt, r1 = -(c + Q xt) into r1
void launch_mehrotra_r1(const IpmDev& d, double* xt, double* r1, cudaStream_t st);
// w = r1 + A'z
void launch_add_atz(const IpmDev& d, const double* r1, double* w, cudaStream_t st);

int reduction_blocks(int n);

}  // namespace sov
