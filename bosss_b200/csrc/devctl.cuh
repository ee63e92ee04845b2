// Device-side control flow of the graph-captured p-multigrid V-cycle.
//
// When the preconditioner is captured as one CUDA graph, every decision the host loop of
// OrthonormalizationMultigrid.Solve takes on a fetched scalar (OrthonormalizationMultigrid.cs:797-1104: the
// termination tests, AddSol's re-orthonormalisation test, MinimizeResidual's residual-increase check, the
// residual period, the history restart) is taken by a one-thread kernel on device state instead, and the loops
// become conditional graph nodes (WHILE for the level's iterations and the coarse CG, IF for the post-smoother
// sweeps, the second Gram-Schmidt sweep and the zero-right-hand-side test of the restriction), whose conditions
// those kernels set.  The history length is a device counter, so the projections use kernels that read it: one
// multi-dot launch and one dual multi-axpy launch whatever the history length.
#pragma once
#include "blas1.cuh"

namespace bsgpu {

// Bits of the device error word of a captured solve (read by the host after the graph).
enum { kDevErrNaN = 1, kDevErrResidualIncrease = 2, kDevErrSlots = 4, kDevErrKrylovNaN = 8 };

// Device state of one OrthonormalizationMultigrid level (CoreOrthonormalizationProcedure + loop).
struct OrthoState {
  int k;        // history length (KrylovDim)
  int cancel;   // the last AddSol dropped its correction (cancellation: nothing new in it)
  int second;   // AddSol needs a second projection sweep
  int recalc;   // the next MinimizeResidual recomputes the residual from scratch ...
  int update;   // ... or updates it (exactly one of the two is set)
  int restart;  // the history was full at the start of this iteration
  int active;   // the level keeps iterating (termination test)
  int iter;     // iteration number, 1-based (iIter of the reference loop)
  int iterations;  // completed iterations (ThisLevelIterations)
  int pad;
  double nM;    // |A x| of the new correction before projection
  double rel;   // |A x| after projection, relative to nM
  double fac;   // scaling of the stored correction (1/|A x| after projection; 0 = dropped)
  double r0, rn;  // initial and current residual norm of the level
};

// Termination parameters of a level (Term, solvers.cuh) passed by value to the decision kernels.
struct TermParams {
  int mode;  // 0: R < R0*tol + tol, 1: R < R0*tol, 2: fixed count, 3: sub-level reduction
  int max_iter, min_iter;
  double tol, reduction;
};

// h = (a == nullptr || *a) && (not_b == nullptr || !*not_b) && (k == nullptr || *k < cap); exec[0] += h.
void cond_set(cudaGraphConditionalHandle h, const int* a, const int* not_b, const int* k, int cap, unsigned int* exec,
              cudaStream_t st);
// flag = (*x > 0)
void positive_flag(const double* x, int* flag, cudaStream_t st);

// beta[j] = <hist[j], m> for j < *k (hist: device array of `cap` vector pointers), self = <m, m> (if self != null);
// one launch.  scratch: partial sums and tickets sized by hist_dots_scratch.
struct HistScratch {
  DBuf<double> partial;
  DBuf<unsigned int> ticket;
  int grid = 0, chunks = 0, slots = 0;  // slots: entries of the pointer arrays (*k is clamped to it)
  void init(int cap);
};
void hist_dots(HistScratch& s, const double* const* hist, const int* k, const double* m, int64_t n, double* beta,
               double* self, cudaStream_t st);
void hist_dots(HistScratch& s, const float* const* hist, const int* k, const float* m, int64_t n, double* beta,
               double* self, cudaStream_t st);
// y1 -= sum_{j<*k} beta[j] x1[j], y2 -= sum_{j<*k} beta[j] x2[j]; one launch (*k clamped to kmax <= kHistMax,
// the entries of the pointer arrays).
constexpr int kHistMax = 128;
void hist_axpy2(const double* const* x1, const double* const* x2, const int* k, int kmax, const double* beta,
                double* y1, double* y2, int64_t n, cudaStream_t st);
void hist_axpy2(const float* const* x1, const float* const* x2, const int* k, int kmax, const double* beta, float* y1,
                float* y2, int64_t n, cudaStream_t st);
// upper bound on the iterations of any recorded loop (a safety bound above every configured limit)
constexpr int kMaxRecordedIterations = 100000;

// AddSol decisions.  proj[0] = |M| after the sweep, proj[1] = |M|^2 before the first sweep.
void ortho_decide1(OrthoState* s, const double* proj, int* err, cudaStream_t st);
void ortho_decide2(OrthoState* s, const double* proj, cudaStream_t st);
void ortho_final(OrthoState* s, const double* proj, cudaStream_t st);
// W *= fac, MW *= fac, and the two stored into history slot *k (slots: device arrays of nslots pointers)
void ortho_store(OrthoState* s, double* W, double* MW, double* const* sol, double* const* mxx, int nslots, int64_t n,
                 int* err, cudaStream_t st);
void ortho_store(OrthoState* s, float* W, float* MW, float* const* sol, float* const* mxx, int nslots, int64_t n,
                 int* err, cudaStream_t st);
// k += 1 (at most nslots) and the residual period decision of the following MinimizeResidual
void ortho_advance(OrthoState* s, int period, int nslots, cudaStream_t st);
// MinimizeResidual's checks on the new residual norm rn_new and the termination test of the level
void minimize_check(OrthoState* s, const double* rn_new, TermParams tp, int* err, cudaStream_t st);
// start of a level solve: r0 = rn = *r0_in, k = 0, iter = 1, iterations = 0, active = term(1, r0, r0)
void level_begin(OrthoState* s, const double* r0_in, TermParams tp, cudaStream_t st);
// start of an iteration: restart = (k >= cap) (then k = 0), cancel = 0
void iter_begin(OrthoState* s, int cap, cudaStream_t st);
// end of an iteration: iterations += active, iter += 1, active = active && term(iter, r0, rn)
void iter_end(OrthoState* s, TermParams tp, cudaStream_t st);
// y -= sum_{j<*k} beta[j] x[j]; one launch (the single-vector form of hist_axpy2)
void hist_axpy1(const double* const* x, const int* k, int kmax, const double* beta, double* y, int64_t n,
                cudaStream_t st);

// Device state of a recorded FlexGMRES solve (FlexGMRES.cs:144-277 with Saad's least-squares update): the
// Arnoldi index, the restart and Arnoldi loop conditions, the round-robin of the two preconditioners and the
// stall fallback of the second, the Givens rotations and the residual history.
struct FgState {
  int j;          // Arnoldi column of the current step
  int k1;         // j + 1: basis vectors the step projects against
  int kk;         // columns of the finished cycle
  int iter;       // preconditioner applications (ThisLevelIterations)
  int outer;      // the restart loop continues
  int inner;      // the Arnoldi loop continues
  int use2;       // this step applies the second preconditioner
  int nn_active;  // the second preconditioner is in use (off after a stall)
  int turn;       // round-robin counter
  int converged;
  int nhist;      // entries written to the residual history
  int stalled;    // the second preconditioner stalled in this solve
  int started;    // r0 is set
  int has2;       // a second preconditioner exists
  int zero;       // constant 0 (slot index of the first basis vector)
  int pad;
  double r0, est, g_before, inv;  // inv: 1/|r| or 1/|w| for the next basis vector (0 when that norm is 0)
};
// Device arrays of the recorded FlexGMRES: Hessenberg matrix (row-major, m columns), rotations, right-hand side
// of the least-squares problem, negated solution, residual history.
struct FgArrays {
  double* H;
  double* cs;
  double* sn;
  double* g;
  double* ny;
  double* hist;
  int m;
  int hcap;
};
// start of a solve: counters cleared, nn_active / has2 as given
void fg_begin(FgState* s, int nn_active, int has2, cudaStream_t st);
// after a residual norm *rn: history, termination test (outer), the first Givens right-hand side g = (r, 0, ...)
void fg_restart(FgState* s, FgArrays a, const double* rn, TermParams tp, int* err, cudaStream_t st);
// start of an Arnoldi step: k1 = j + 1, which preconditioner it applies, |g_j| before it
void fg_step_begin(FgState* s, FgArrays a, cudaStream_t st);
// end of an Arnoldi step: Hessenberg column from the two projection sweeps h1, h2 and |w|, Givens rotation,
// residual estimate, stall test of the second preconditioner, termination test (inner), j += 1
void fg_step_end(FgState* s, FgArrays a, const double* h1, const double* h2, const double* wn, TermParams tp,
                 double stall, int* err, cudaStream_t st);
// back substitution of the finished cycle: ny = -H^{-1} g (kk columns)
void fg_backsub(FgState* s, FgArrays a, cudaStream_t st);
// out = tab[*idx] (idx null: slot 0)
void slot_load(const double* const* tab, const int* idx, double* out, int64_t n, cudaStream_t st);
// tab[*idx] = x * (*scale) (scale null: 1); an index outside 0..nslots-1 sets kDevErrSlots
void slot_store(const double* x, const double* scale, double* const* tab, const int* idx, int nslots, int64_t n,
                int* err, cudaStream_t st);

// dst[i][0..n[i]) = src[i][0..n[i]) for i < count (the staging copies of a batch, one launch)
void batch_copy(const double* const* src, double* const* dst, const int64_t* n, int count, cudaStream_t st);

// y = x where *flag (vector copy predicated on a device flag)
void copy_if(const double* x, double* y, int64_t n, const int* flag, cudaStream_t st);
void copy_if(const float* x, float* y, int64_t n, const int* flag, cudaStream_t st);

}  // namespace bsgpu
