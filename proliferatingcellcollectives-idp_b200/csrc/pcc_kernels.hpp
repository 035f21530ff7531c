// Host launchers of the device kernels (internal to libpcc_gpu.so).
#pragma once

#include <cuda_runtime.h>

#include "pcc_ctx.hpp"

namespace pcc {

// Slots of ctx->pinned_ll for values copied back at a synchronisation point
// (slots 0..7 belong to the detection pass).
constexpr int kSlotMedian = 8;   // two adaptDt median keys
constexpr int kSlotRadius = 10;  // colony radius bits
constexpr int kSlotDivs = 11;    // divisions of the next step
constexpr int kSlotMaxOld = 12;  // largest overlap of the earlier phases' constraints

// ---- pcc_scan_sort.cu
// out[i] = sum in[0..i-1] for i in [0, n]; out has n+1 entries.
cudaError_t exclusive_scan(pcc_ctx* ctx, const int* in, int* out, size_t n);
// Stable ascending sort of (keys, vals) by the low `bits` bits of keys;
// keys/vals are sorted in place (scratch from ctx).
cudaError_t radix_sort_pairs(pcc_ctx* ctx, unsigned long long* keys, int* vals, size_t n, int bits);

// ---- pcc_detect.cu
// Appends the contacts within tol of the resident cells to the constraint set
// (ctx->ncons grows by *added).  *max_overlap_new = max(-sd, 0) over them.
// reuse = true lets a later ReLCP phase of the same step re-test the
// candidate lists of the previous full pass instead of rebinning; callers
// pass it only when the cells changed by constraint motion alone since.
cudaError_t detect_contacts(pcc_ctx* ctx, double tol, int phase, bool reuse, size_t* added,
                            double* max_overlap_new);
// Cell -> incident constraint sides, ascending constraint index, for ctx->ncons.
cudaError_t build_incidence(pcc_ctx* ctx);

// ---- pcc_solver.cu
// Draws the Brownian U_ext of every cell (temperature > 0) from the context's
// generator and sets ctx->uext_active; a no-op at temperature 0.
cudaError_t brownian_draw(pcc_ctx* ctx);
// One BBPGD solve on the current constraint set (hard model).  With defer,
// only launches it and enqueues the copy of its scalars (ctx->bbpgd_pending);
// bbpgd_collect reads them after the caller's next synchronisation.
cudaError_t bbpgd_solve(pcc_ctx* ctx, double dt, long long* iterations, double* residual, int* status,
                        bool defer = false);
void bbpgd_collect(pcc_ctx* ctx, long long* iterations, double* residual, int* status);
// Largest overlap of constraints [from, to) into ctx->pinned_ll[kSlotMaxOld]
// at the next synchronisation (no host wait).
cudaError_t max_overlap_enqueue(pcc_ctx* ctx, size_t from, size_t to);
// Moves cells with the solver's velocities and writes back gamma / phi.
cudaError_t apply_hard_solution(pcc_ctx* ctx, double dt);
// Soft model: Hertz forces, motion and growth parameters.
cudaError_t soft_forces_and_move(pcc_ctx* ctx, double dt);
// Soft model force assembly only (frozen microbench).
cudaError_t soft_assemble(pcc_ctx* ctx);

// ---- pcc_planar.cu
// BBPGD trace buffers handed to the planar solver (trace = 0: none).
struct PlanarTrace {
  int trace;
  double* tr_part;
  double* trace_out;
  long long trace_cap;
};
// Constraint chunks of the planar solver's reductions for m constraints.
long long planar_chunks(size_t m);
// Packs the planar operands and launches the planar BBPGD solve on the
// context's stream (FP64, or mixed precision); *kind = 1 for the multi-block
// cooperative kernel, 0 for a one-block launch.
cudaError_t planar_bbpgd(pcc_ctx* ctx, double dt, bool mixed, const PlanarTrace& tr, int* kind);

// ---- pcc_update.cu
cudaError_t reset_ldot(pcc_ctx* ctx);
cudaError_t grow_cells(pcc_ctx* ctx, double dt);
// Division of every cell with len >= 2 l0, daughters appended; returns count.
// Uses the flags counted at the end of the previous step when ctx->div_known.
cudaError_t divide_cells(pcc_ctx* ctx, size_t* added);
// End-of-step work whose results come back in one copy: the division flags
// and count of the next step, the colony radius, the adaptDt median keys.
cudaError_t division_count_enqueue(pcc_ctx* ctx);
cudaError_t radius_enqueue(pcc_ctx* ctx);
double radius_collect(pcc_ctx* ctx);
cudaError_t adapt_dt_enqueue(pcc_ctx* ctx);
void adapt_dt_collect(pcc_ctx* ctx);  // updates ctx->params.dt
// Sort cells by x (stable) and renumber.
cudaError_t sort_cells_by_x(pcc_ctx* ctx);
cudaError_t colony_radius(pcc_ctx* ctx, double* out);
cudaError_t adapt_dt(pcc_ctx* ctx);  // updates ctx->params.dt
cudaError_t mobility(pcc_ctx* ctx);

// ---- pcc_vtk.cu
// Waits for and stops the context's VTK writer thread.
void vtk_writer_shutdown(pcc_ctx* ctx);
// Removes <dir>/<prefix>*.pvtu and <dir>/data/<prefix>*.vtu (a new logger's reset).
void vtk_clear_prefix(const std::string& dir, const std::string& prefix);
// bbpgdtrace_<index> files of BBPGDLogger::log, indices first_index, first_index + 1, ...
bool vtk_write_trace(const std::string& dir, unsigned long long first_index,
                     const std::vector<pcc_bbpgd_trace_step>& steps);

}  // namespace pcc
