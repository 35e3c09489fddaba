// FP64 BiCGStab solvers with the reference's algorithm, update order and
// stopping rule: invert_Qtm (BiCGStab on Q, invert_Qtm.c:86-270) and
// invert_Qtm_her (BiCGStab on Qf5(mu) Qf5(-mu) with right-hand side g5 phi,
// then x = Qf5(-mu) y, invert_Qtm.c:276-478).
//
// The recursion scalars live on the device (SolverScalars): the last block of
// each reduction computes alpha, omega, beta and the convergence flag, and
// every later kernel of the iteration reads them from HBM.  An iteration thus
// costs no host round trip; the host checks the flag once per chunk of
// iterations.  Once the flag is set, all remaining kernels of the chunk
// return immediately, so the state is exactly that of the iteration at which
// the reference would have left its loop.
#include <algorithm>
#include <cmath>

#include "cvcb_internal.h"
#include "reduce.cuh"

namespace cvcb {

namespace {

__device__ __forceinline__ double2 c_div(double2 a, double2 b) {
  // _co_eq_co_ti_co_inv (cvc_complex.h): a / b = a conj(b) / |b|^2
  const double n = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / n, (a.y * b.x - a.x * b.y) / n);
}
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ bool finite2(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// rho = <r2, r1>, w = <r2, p2>; alpha = rho / w  (invert_Qtm.c:161-163)
struct RedRhoW {
  const double2 *r2, *r1, *p2;
  __device__ void operator()(size_t k, double (&acc)[4]) const {
    const double2 a = __ldg(r2 + k), b = __ldg(r1 + k), c = __ldg(p2 + k);
    acc[0] += a.x * b.x + a.y * b.y;
    acc[1] += a.x * b.y - a.y * b.x;
    acc[2] += a.x * c.x + a.y * c.y;
    acc[3] += a.x * c.y - a.y * c.x;
  }
};
struct EpiAlpha {
  SolverScalars *S;
  __device__ void operator()(const double (&t)[4]) const {
    S->rho = make_double2(t[0], t[1]);
    S->w = make_double2(t[2], t[3]);
    S->alpha = c_div(S->rho, S->w);
    if (!finite2(S->alpha)) { S->done = 2; S->niter = S->iter; }
  }
};

// s = r1 - alpha p2   (invert_Qtm.c:171-176)
__global__ void k_s_update(double2 *__restrict__ s, const double2 *__restrict__ r1,
                           const double2 *__restrict__ p2, const SolverScalars *__restrict__ S,
                           size_t n) {
  if (S->done) return;
  const double2 al = S->alpha;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const double2 q = c_mul(__ldg(p2 + k), al);
    const double2 r = __ldg(r1 + k);
    s[k] = make_double2(r.x - q.x, r.y - q.y);
  }
}

// w = <t, s>, u = <t, t>; omega = w / u  (invert_Qtm.c:182-184)
struct RedOmega {
  const double2 *t, *s;
  __device__ void operator()(size_t k, double (&acc)[3]) const {
    const double2 a = __ldg(t + k), b = __ldg(s + k);
    acc[0] += a.x * b.x + a.y * b.y;
    acc[1] += a.x * b.y - a.y * b.x;
    acc[2] += a.x * a.x + a.y * a.y;
  }
};
struct EpiOmega {
  SolverScalars *S;
  __device__ void operator()(const double (&t)[3]) const {
    S->u = t[2];
    // invert_Qtm.c:184 writes _co_eq_co_ti_re(&omega, &w, 1./u); the macro
    // argument is not parenthesised, so it evaluates w.re*1./u = w.re / u.
    S->omega = make_double2(t[0] / S->u, t[1] / S->u);
    if (!finite2(S->omega)) { S->done = 2; S->niter = S->iter; }
  }
};

// r1 = s - omega t; norm = <r1, r1>; stop if norm <= prec * normb
// (invert_Qtm.c:192-201).
struct RedR1 {
  double2 *r1;
  const double2 *s, *t;
  const SolverScalars *S;
  __device__ void operator()(size_t k, double (&acc)[1]) const {
    const double2 q = c_mul(__ldg(t + k), S->omega);
    const double2 a = __ldg(s + k);
    const double2 r = make_double2(a.x - q.x, a.y - q.y);
    r1[k] = r;
    acc[0] += r.x * r.x + r.y * r.y;
  }
};
struct EpiNorm {
  SolverScalars *S;
  __device__ void operator()(const double (&t)[1]) const {
    S->norm = t[0];
    if (S->norm <= S->prec * S->normb) {
      S->done = 1;
      S->niter = S->iter;
    } else if (!isfinite(S->norm)) {
      S->done = 2;
      S->niter = S->iter;
    }
  }
};

// x += omega s + alpha p; w = <r2, r1>; beta = (w / rho)(alpha / omega);
// rho = w  (invert_Qtm.c:204-218).  Skipped once converged: the reference
// leaves the loop before this update.
struct RedXBeta {
  double2 *x;
  const double2 *s, *p, *r2, *r1;
  const SolverScalars *S;
  __device__ void operator()(size_t k, double (&acc)[2]) const {
    double2 xv = x[k];
    const double2 a = c_mul(__ldg(s + k), S->omega);
    xv.x += a.x; xv.y += a.y;
    const double2 b = c_mul(__ldg(p + k), S->alpha);
    xv.x += b.x; xv.y += b.y;
    x[k] = xv;
    const double2 u = __ldg(r2 + k), v = __ldg(r1 + k);
    acc[0] += u.x * v.x + u.y * v.y;
    acc[1] += u.x * v.y - u.y * v.x;
  }
};
struct EpiBeta {
  SolverScalars *S;
  __device__ void operator()(const double (&t)[2]) const {
    const double2 w = make_double2(t[0], t[1]);
    const double2 w2 = c_div(w, S->rho);
    const double2 w3 = c_div(S->alpha, S->omega);
    S->beta = c_mul(w2, w3);
    S->rho = w;
    S->iter += 1;
    if (!finite2(S->beta)) { S->done = 2; S->niter = S->iter; }
  }
};

// p = r1 + beta (p - omega p2)  (invert_Qtm.c:224-231)
__global__ void k_p_update(double2 *__restrict__ p, const double2 *__restrict__ r1,
                           const double2 *__restrict__ p2, const SolverScalars *__restrict__ S,
                           size_t n) {
  if (S->done) return;
  const double2 om = S->omega, be = S->beta;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const double2 q = c_mul(__ldg(p2 + k), om);
    const double2 pv = p[k];
    const double2 d = make_double2(pv.x - q.x, pv.y - q.y);
    const double2 e = c_mul(d, be);
    const double2 r = __ldg(r1 + k);
    p[k] = make_double2(r.x + e.x, r.y + e.y);
  }
}

// y = a - b
__global__ void k_sub(double2 *__restrict__ y, const double2 *__restrict__ a,
                      const double2 *__restrict__ b, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const double2 u = __ldg(a + k), v = __ldg(b + k);
    y[k] = make_double2(u.x - v.x, u.y - v.y);
  }
}

struct RedNorm {
  const double2 *a;
  __device__ void operator()(size_t k, double (&acc)[1]) const {
    const double2 u = __ldg(a + k);
    acc[0] += u.x * u.x + u.y * u.y;
  }
};

struct EpiNormb {
  SolverScalars *S;
  __device__ void operator()(const double (&t)[1]) const { S->normb = t[0]; }
};
struct EpiStart {
  SolverScalars *S;
  __device__ void operator()(const double (&t)[1]) const {
    S->norm = t[0];
    if (S->norm <= S->prec * S->normb) { S->done = 3; S->niter = 0; }
  }
};

int elem_blocks(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 4096 ? 4096 : b);
}

}  // namespace

// The operator of each solver on device-layout FP64 fields.
static int apply_op(cvcb_lattice *L, bool her, double2 *out, const double2 *in, double2 *aux,
                    const int *done) {
  const double a = 0.5 / L->kappa;
  if (!her) return launch_tm_full(L, out, in, a, L->mu, -0.5, false, done);
  CVCB_TRY(launch_tm_full(L, aux, in, a, -L->mu, -0.5, true, done));  // Qf5(aux, in, -mu)
  return launch_tm_full(L, out, aux, a, L->mu, -0.5, true, done);     // Qf5(out, aux, +mu)
}

int invert_bicgstab(cvcb_lattice *L, bool her, double *xi, const double *phi, double prec,
                    int niter_max, double *true_res2) {
  const Geom &g = L->g;
  const size_t n = (size_t)g.V * 12;
  const size_t fb = n * sizeof(double2);
  void *base;
  CVCB_TRY(ensure_buffer(L, SLOT_F2, 10 * fb, &base));
  double2 *F = static_cast<double2 *>(base);
  double2 *x = F, *rhs = F + n, *r1 = F + 2 * n, *r2 = F + 3 * n, *s = F + 4 * n,
          *t = F + 5 * n, *p = F + 6 * n, *p2 = F + 7 * n, *aux = F + 8 * n, *phid = F + 9 * n;
  SolverScalars *S = L->scal;
  const int eb = elem_blocks(n);

  CVCB_TRY(spinor_in(L, phid, phi, g.V));
  CVCB_TRY(spinor_in(L, x, xi, g.V));

  SolverScalars h{};
  h.prec = prec;
  CVCB_CUDA(cudaMemcpyAsync(S, &h, sizeof h, cudaMemcpyHostToDevice, L->stream));

  // normb = <phi, phi>  (invert_Qtm.c:129 / :329)
  CVCB_TRY(launch_reduce<1>(L, RedNorm{phid}, EpiNormb{S}, n));
  if (her) {
    CVCB_CUDA(cudaMemcpyAsync(rhs, phid, fb, cudaMemcpyDeviceToDevice, L->stream));
    CVCB_TRY(launch_g5(L, rhs, g.V));
  } else {
    rhs = phid;
  }
  // p = rhs - A x ; norm = <p,p>
  CVCB_TRY(apply_op(L, her, p, x, aux, nullptr));
  k_sub<<<eb, 256, 0, L->stream>>>(p, rhs, p, n);
  CVCB_LAUNCHED(L);
  CVCB_TRY(launch_reduce<1>(L, RedNorm{p}, EpiStart{S}, n));
  SolverScalars hs;
  CVCB_CUDA(cudaMemcpyAsync(&hs, S, sizeof hs, cudaMemcpyDeviceToHost, L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  if (hs.done == 3) {
    // start guess already solves: the reference returns 0 and leaves xi as
    // it was (invert_Qtm.c:144-147, :344-347).
    if (true_res2) *true_res2 = hs.norm / hs.normb;
    return 0;
  }

  CVCB_CUDA(cudaMemcpyAsync(r1, p, fb, cudaMemcpyDeviceToDevice, L->stream));
  CVCB_CUDA(cudaMemcpyAsync(r2, p, fb, cudaMemcpyDeviceToDevice, L->stream));
  CVCB_TRY(apply_op(L, her, p2, p, aux, nullptr));

  const int *done = &S->done;
  const int chunk = 16;
  int launched = 0;
  for (;;) {
    const int todo = std::min(chunk, niter_max + 1 - launched);
    for (int it = 0; it < todo; ++it) {
      CVCB_TRY(launch_reduce<4>(L, RedRhoW{r2, r1, p2}, EpiAlpha{S}, n, done));
      k_s_update<<<eb, 256, 0, L->stream>>>(s, r1, p2, S, n);
      CVCB_LAUNCHED(L);
      CVCB_TRY(apply_op(L, her, t, s, aux, done));
      CVCB_TRY(launch_reduce<3>(L, RedOmega{t, s}, EpiOmega{S}, n, done));
      CVCB_TRY(launch_reduce<1>(L, RedR1{r1, s, t, S}, EpiNorm{S}, n, done));
      CVCB_TRY(launch_reduce<2>(L, RedXBeta{x, s, p, r2, r1, S}, EpiBeta{S}, n, done));
      k_p_update<<<eb, 256, 0, L->stream>>>(p, r1, p2, S, n);
      CVCB_LAUNCHED(L);
      CVCB_TRY(apply_op(L, her, p2, p, aux, done));
    }
    launched += todo;
    CVCB_CUDA(cudaMemcpyAsync(&hs, S, sizeof hs, cudaMemcpyDeviceToHost, L->stream));
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
    if (hs.done || launched > niter_max) break;
  }
  const int niter = hs.done == 1 ? hs.niter : niter_max + 1;
  const bool converged = hs.done == 1 && niter <= niter_max;

  if (her) {
    // x = Qf5(x, -mu)  (invert_Qtm.c:443-446), done whether or not converged
    CVCB_TRY(launch_tm_full(L, aux, x, 0.5 / L->kappa, -L->mu, -0.5, true, nullptr));
    std::swap(x, aux);
  }
  CVCB_TRY(spinor_out(L, xi, x, g.V));
  if (!converged) {
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
    if (hs.done == 2) {  // a non-finite alpha, omega or beta stopped the recursion
      set_error("BiCGStab broke down after %d iterations (relative residual^2 %g)", hs.niter,
                hs.norm / hs.normb);
      return CVCB_BREAKDOWN;
    }
    set_error("no convergence after %d iterations (relative residual^2 %g)", niter,
              hs.norm / hs.normb);
    return CVCB_NO_CONVERGENCE;
  }
  if (true_res2) {
    // true residual |Q x - phi|^2 / |phi|^2 (invert_Qtm.c:257-267 / :466-475)
    CVCB_TRY(launch_tm_full(L, t, x, 0.5 / L->kappa, L->mu, -0.5, false, nullptr));
    k_sub<<<eb, 256, 0, L->stream>>>(t, t, phid, n);
    CVCB_LAUNCHED(L);
    double r2n;
    CVCB_TRY(dot_re(L, t, t, n, &r2n));
    *true_res2 = r2n / hs.normb;
  }
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return niter;
}

}  // namespace cvcb

extern "C" {

int cvcb_invert_Qtm(cvcb_lattice *L, double *xi, const double *phi, double solver_precision,
                    int niter_max, double *true_res2) {
  if (!L || !xi || !phi) return CVCB_ERR_NULL;
  if (!L->have_gauge) {
    cvcb::set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::invert_bicgstab(L, false, xi, phi, solver_precision, niter_max, true_res2);
}

int cvcb_invert_Qtm_her(cvcb_lattice *L, double *xi, const double *phi, double solver_precision,
                        int niter_max, double *true_res2) {
  if (!L || !xi || !phi) return CVCB_ERR_NULL;
  if (!L->have_gauge) {
    cvcb::set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::invert_bicgstab(L, true, xi, phi, solver_precision, niter_max, true_res2);
}

}  // extern "C"
