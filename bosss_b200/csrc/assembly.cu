// SIP (symmetric interior penalty) DG discretisation of -div(nu grad u) on a uniform Cartesian grid, assembled on
// the GPU straight into block-CSR form: the operator the solver path takes, without the host assembly of
// ipLaplace.cs (volume term :95-130, inner-edge terms :150-200, boundary terms :205-245) and its transfer.
//
// Basis: per cell the orthonormal Legendre products of total degree <= p, modes ordered by total degree, then
// lexicographically by exponent tuple (the order of the reference's hierarchical basis, so p-restriction keeps the
// leading modes).  On a uniform grid every block is a linear combination of a few Np x Np templates (the 1-D
// volume, trace and normal-derivative matrices of direction d, expanded with the Kronecker delta in the other
// directions) whose coefficients depend only on the diffusivities and length scales of the cells beside a face:
//   inner face between L and R = L + e_d:  eta = penalty * max(cj_L, cj_R) * max(nu_L, nu_R),
//   boundary face (homogeneous Dirichlet):  eta = 2 * penalty * cj * nu,
//   cj = 0.5 * (surface + boundary area) / volume  (GridData_CellData.cs:681-687).
// The host computes the templates (Gauss-Legendre quadrature of the 1-D stiffness matrix, traces at +-1); one thread
// per block entry keeps its entries of all templates in registers and writes that entry of every block of a range of
// cells (coalesced: the threads of a CTA write whole blocks).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

#include "matrix.cuh"

namespace bsgpu {

namespace {

// orthonormal Legendre psi_n(t) = sqrt((2n+1)/2) P_n(t) and its derivative, by the three-term recurrences
// P_{n+1} = ((2n+1) t P_n - n P_{n-1}) / (n+1) and P'_{n+1} = P'_{n-1} + (2n+1) P_n
void legendre_all(int pmax, double t, std::vector<double>& P, std::vector<double>& dP) {
  P.assign(pmax + 1, 0.0);
  dP.assign(pmax + 1, 0.0);
  P[0] = 1.0;
  if (pmax >= 1) {
    P[1] = t;
    dP[1] = 1.0;
  }
  for (int n = 1; n < pmax; ++n) {
    P[n + 1] = ((2.0 * n + 1.0) * t * P[n] - n * P[n - 1]) / (n + 1.0);
    dP[n + 1] = dP[n - 1] + (2.0 * n + 1.0) * P[n];
  }
  for (int n = 0; n <= pmax; ++n) {
    const double s = std::sqrt((2.0 * n + 1.0) / 2.0);
    P[n] *= s;
    dP[n] *= s;
  }
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_q from the Chebyshev guesses)
void gauss_legendre(int q, std::vector<double>& x, std::vector<double>& w) {
  x.assign(q, 0.0);
  w.assign(q, 0.0);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < q; ++i) {
    double t = std::cos(pi * (i + 0.75) / (q + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = t;
      for (int n = 1; n < q; ++n) {
        const double p2 = ((2.0 * n + 1.0) * t * p1 - n * p0) / (n + 1.0);
        p0 = p1;
        p1 = p2;
      }
      const double pq = q == 0 ? 1.0 : (q == 1 ? t : p1);
      const double pqm1 = q == 1 ? 1.0 : p0;
      dp = q * (t * pq - pqm1) / (t * t - 1.0);
      const double dt = pq / dp;
      t -= dt;
      if (std::fabs(dt) < 1e-16) break;
    }
    x[i] = t;
    w[i] = 2.0 / ((1.0 - t * t) * dp * dp);
  }
}

std::vector<std::array<int, 3>> modes_of(int D, int p) {
  std::vector<std::array<int, 3>> out;
  for (int deg = 0; deg <= p; ++deg) {
    if (D == 1) {
      out.push_back({deg, 0, 0});
    } else if (D == 2) {
      for (int i = 0; i <= deg; ++i) out.push_back({i, deg - i, 0});
    } else {
      for (int i = 0; i <= deg; ++i)
        for (int j = 0; j <= deg - i; ++j) out.push_back({i, j, deg - i - j});
    }
  }
  return out;
}

// Template indices: 0 volume; per direction d (base 1 + 4d): A = -(t d^T + d t^T)/2 at +1, B = t t^T at +1,
// C = (t d^T + d t^T)/2 at -1, E = t t^T at -1; off-diagonal per direction (base 1 + 4D + 6d): P = -t(+1) d(-1)^T/2,
// Q = d(+1) t(-1)^T/2, R = -t(+1) t(-1)^T and their transposes.
constexpr int kMaxD = 3;
constexpr int kTemplates = 1 + 4 * kMaxD + 6 * kMaxD;

struct SipArgs {
  int D;
  int n[kMaxD];
  int64_t stride[kMaxD];
  double hinv[kMaxD];  // 1 / h_d
  double penalty;
  int Np;
  int64_t nc;
};

__device__ __forceinline__ double cj_of(const SipArgs& a, const int (&idx)[kMaxD]) {
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < kMaxD; ++d) {
    if (d >= a.D) break;
    const int nbnd = (idx[d] == 0 ? 1 : 0) + (idx[d] == a.n[d] - 1 ? 1 : 0);
    s += (2.0 + nbnd) * a.hinv[d];
  }
  return 0.5 * s;
}

// One CTA per range of cells; thread v owns entry v of every block.  rp: block-row offsets (ascending block
// columns per row: -z, -y, -x, self, +x, +y, +z as present).
__global__ void sip_assemble_kernel(SipArgs a, const double* __restrict__ tmpl, const double* __restrict__ nu,
                                    const int64_t* __restrict__ rp, double* __restrict__ vals) {
  const int NN = a.Np * a.Np;
  const int v = threadIdx.x;
  if (v >= NN) return;
  double T[kTemplates];
#pragma unroll
  for (int t = 0; t < kTemplates; ++t) T[t] = tmpl[(int64_t)t * NN + v];
  // entry v of the transposed off-diagonal templates: index (col, row)
  const int vr = v / a.Np, vc = v - (v / a.Np) * a.Np;
  const int vt = vc * a.Np + vr;
  double TT[3 * kMaxD];
#pragma unroll
  for (int d = 0; d < kMaxD; ++d)
#pragma unroll
    for (int q = 0; q < 3; ++q) TT[3 * d + q] = tmpl[(int64_t)(1 + 4 * kMaxD + 6 * d + q) * NN + vt];
  for (int64_t c = blockIdx.x; c < a.nc; c += gridDim.x) {
    int idx[kMaxD] = {0, 0, 0};
    int64_t rem = c;
#pragma unroll
    for (int d = 0; d < kMaxD; ++d) {
      idx[d] = (int)(rem % a.n[d]);  // n[d] = 1 for d >= D
      rem /= a.n[d];
    }
    const double kc = nu ? nu[c] : 1.0;
    const double cjc = cj_of(a, idx);
    double diag = kc * T[0];
    int64_t slot = rp[c];
    // lower neighbours (-z, -y, -x) come first (loops over kMaxD, unrolled, so the template indices are constants)
#pragma unroll
    for (int d = kMaxD - 1; d >= 0; --d) {
      if (d >= a.D || idx[d] == 0) continue;
      const int64_t L = c - a.stride[d];
      int il[kMaxD] = {idx[0], idx[1], idx[2]};
      il[d] -= 1;
      const double kL = nu ? nu[L] : 1.0;
      const double eta = a.penalty * fmax(cj_of(a, il), cjc) * fmax(kL, kc);
      // row c (the right cell R of the face), column L: kR P^T + kL Q^T + eta R^T with R = c
      vals[slot * NN + v] = kc * TT[3 * d] + kL * TT[3 * d + 1] + eta * TT[3 * d + 2];
      ++slot;
    }
    // diagonal: volume + the -d side (templates C, E) and the +d side (A, B) of every direction
#pragma unroll
    for (int d = 0; d < kMaxD; ++d) {
      if (d >= a.D) continue;
      const int base = 1 + 4 * d;
      // +d side
      if (idx[d] < a.n[d] - 1) {
        int ir[kMaxD] = {idx[0], idx[1], idx[2]};
        ir[d] += 1;
        const double kR = nu ? nu[c + a.stride[d]] : 1.0;
        const double eta = a.penalty * fmax(cjc, cj_of(a, ir)) * fmax(kc, kR);
        diag += kc * T[base] + eta * T[base + 1];
      } else {
        diag += 2.0 * kc * T[base] + 2.0 * a.penalty * cjc * kc * T[base + 1];
      }
      // -d side
      if (idx[d] > 0) {
        int il[kMaxD] = {idx[0], idx[1], idx[2]};
        il[d] -= 1;
        const double kL = nu ? nu[c - a.stride[d]] : 1.0;
        const double eta = a.penalty * fmax(cj_of(a, il), cjc) * fmax(kL, kc);
        diag += kc * T[base + 2] + eta * T[base + 3];
      } else {
        diag += 2.0 * kc * T[base + 2] + 2.0 * a.penalty * cjc * kc * T[base + 3];
      }
    }
    vals[slot * NN + v] = diag;
    ++slot;
    // upper neighbours (+x, +y, +z)
#pragma unroll
    for (int d = 0; d < kMaxD; ++d) {
      if (d >= a.D || idx[d] == a.n[d] - 1) continue;
      const int64_t R = c + a.stride[d];
      int ir[kMaxD] = {idx[0], idx[1], idx[2]};
      ir[d] += 1;
      const double kR = nu ? nu[R] : 1.0;
      const double eta = a.penalty * fmax(cjc, cj_of(a, ir)) * fmax(kc, kR);
      const int ob = 1 + 4 * kMaxD + 6 * d;
      // row c (the left cell L of the face), column R: kR P + kL Q + eta R with L = c
      vals[slot * NN + v] = kR * T[ob] + kc * T[ob + 1] + eta * T[ob + 2];
      ++slot;
    }
  }
}

}  // namespace

std::vector<double> sip_templates(int D, int p, const double* h) {
  require(D >= 1 && D <= 3, "D must be 1, 2 or 3");
  require(p >= 0 && p <= 6, "p must be in 0..6");
  const auto modes = modes_of(D, p);
  const int Np = (int)modes.size();
  std::vector<double> gx, gw, P, dP;
  gauss_legendre(p + 2, gx, gw);
  std::vector<double> S((p + 1) * (p + 1), 0.0);
  for (size_t g = 0; g < gx.size(); ++g) {
    legendre_all(p, gx[g], P, dP);
    for (int m = 0; m <= p; ++m)
      for (int n = 0; n <= p; ++n) S[m * (p + 1) + n] += gw[g] * dP[m] * dP[n];
  }
  std::vector<double> Pp, dPp, Pm, dPm;
  legendre_all(p, 1.0, Pp, dPp);
  legendre_all(p, -1.0, Pm, dPm);
  const int NN = Np * Np;
  std::vector<double> T((size_t)kTemplates * NN, 0.0);
  auto expand = [&](int tid, int d, auto&& f) {
    for (int r = 0; r < Np; ++r)
      for (int c = 0; c < Np; ++c) {
        bool same = true;
        for (int e = 0; e < D; ++e)
          if (e != d && modes[r][e] != modes[c][e]) same = false;
        if (same) T[(size_t)tid * NN + r * Np + c] += f(modes[r][d], modes[c][d]);
      }
  };
  for (int d = 0; d < D; ++d) {
    require(h[d] > 0, "cell sizes must be positive");
    const double hd = h[d];
    const double s = std::sqrt(2.0 / hd);  // traces: sqrt(2/h) psi(+-1); normal derivatives: sqrt(2/h) (2/h) psi'
    const double ds = s * 2.0 / hd;
    auto tp = [&](int m) { return s * Pp[m]; };
    auto dp = [&](int m) { return ds * dPp[m]; };
    auto tm = [&](int m) { return s * Pm[m]; };
    auto dm = [&](int m) { return ds * dPm[m]; };
    expand(0, d, [&](int m, int n) { return 4.0 / (hd * hd) * S[m * (p + 1) + n]; });
    const int b = 1 + 4 * d;
    expand(b, d, [&](int m, int n) { return -0.5 * (tp(m) * dp(n) + dp(m) * tp(n)); });
    expand(b + 1, d, [&](int m, int n) { return tp(m) * tp(n); });
    expand(b + 2, d, [&](int m, int n) { return 0.5 * (tm(m) * dm(n) + dm(m) * tm(n)); });
    expand(b + 3, d, [&](int m, int n) { return tm(m) * tm(n); });
    const int ob = 1 + 4 * kMaxD + 6 * d;
    expand(ob, d, [&](int m, int n) { return -0.5 * tp(m) * dm(n); });
    expand(ob + 1, d, [&](int m, int n) { return 0.5 * dp(m) * tm(n); });
    expand(ob + 2, d, [&](int m, int n) { return -tp(m) * tm(n); });
  }
  return T;
}

int sip_template_count() { return kTemplates; }

int modes_count(int D, int p) {
  require(D >= 1 && D <= 3 && p >= 0, "D must be 1, 2 or 3 and p >= 0");
  return (int)modes_of(D, p).size();
}

Matrix* assemble_sip_cartesian(int D, const int32_t* shape, double lo, double hi, int p, double penalty,
                               const double* nu, bool nu_device) {
  require(D >= 1 && D <= 3, "D must be 1, 2 or 3");
  require(p >= 0 && p <= 6, "p must be in 0..6");
  require(hi > lo, "the box must have hi > lo");
  require(penalty > 0, "the penalty factor must be positive");
  int64_t nc = 1;
  SipArgs a{};
  a.D = D;
  for (int d = 0; d < kMaxD; ++d) {
    a.n[d] = 1;
    a.stride[d] = 0;
  }
  for (int d = 0; d < D; ++d) {
    require(shape[d] >= 1, "every grid extent must be >= 1");
    a.n[d] = shape[d];
    a.stride[d] = nc;
    a.hinv[d] = shape[d] / (hi - lo);
    nc *= shape[d];
  }
  a.nc = nc;
  a.penalty = penalty;
  const auto modes = modes_of(D, p);
  const int Np = (int)modes.size();
  a.Np = Np;
  require(Np * Np <= 1024, "blocks above 32 x 32 entries are not supported");
  double hs[kMaxD] = {1.0, 1.0, 1.0};
  for (int d = 0; d < D; ++d) hs[d] = 1.0 / a.hinv[d];
  const std::vector<double> T = sip_templates(D, p, hs);
  const int NN = Np * Np;
  // structure: block columns ascending per row (-z, -y, -x, self, +x, +y, +z as present)
  std::vector<int64_t> rp(nc + 1, 0);
  std::vector<int32_t> ci;
  ci.reserve((size_t)nc * (2 * D + 1));
  for (int64_t c = 0; c < nc; ++c) {
    int idx[kMaxD] = {0, 0, 0};
    int64_t rem = c;
    for (int d = 0; d < D; ++d) {
      idx[d] = (int)(rem % a.n[d]);
      rem /= a.n[d];
    }
    for (int d = D - 1; d >= 0; --d)
      if (idx[d] > 0) ci.push_back((int32_t)(c - a.stride[d]));
    ci.push_back((int32_t)c);
    for (int d = 0; d < D; ++d)
      if (idx[d] < a.n[d] - 1) ci.push_back((int32_t)(c + a.stride[d]));
    rp[c + 1] = (int64_t)ci.size();
  }
  require(nc < (int64_t)INT32_MAX, "too many cells");
  const int64_t nnzb = (int64_t)ci.size();
  DBuf<double> d_t(T.size()), d_vals((size_t)std::max<int64_t>(nnzb, 1) * NN), d_nu;
  DBuf<int64_t> d_rp(nc + 1);
  DBuf<int32_t> d_ci(std::max<int64_t>(nnzb, 1));
  BSGPU_CUDA(cudaMemcpy(d_t.p, T.data(), T.size() * 8, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(d_rp.p, rp.data(), (nc + 1) * 8, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(d_ci.p, ci.data(), nnzb * 4, cudaMemcpyHostToDevice));
  const double* nu_dev = nullptr;
  if (nu) {
    if (nu_device) {
      nu_dev = nu;
    } else {
      d_nu.alloc(nc);
      BSGPU_CUDA(cudaMemcpy(d_nu.p, nu, nc * 8, cudaMemcpyHostToDevice));
      nu_dev = d_nu.p;
    }
  }
  const int threads = ((NN + 31) / 32) * 32;
  const int grid = (int)std::min<int64_t>(nc, (int64_t)num_sms() * 16);
  sip_assemble_kernel<<<grid, threads>>>(a, d_t.p, nu_dev, d_rp.p, d_vals.p);
  BSGPU_CHECK_LAUNCH();
  BSGPU_CUDA(cudaDeviceSynchronize());
  return matrix_create(nc, Np, nullptr, d_rp.p, d_ci.p, d_vals.p, BSGPU_DEVICE_POINTERS);
}

}  // namespace bsgpu

namespace bsgpu {

namespace {

// out[c * Np + a] = sum_m coef[m] prod_d T[((m * D + d) * nmax + i_d(c)) * (p + 1) + mode_a[d]]
__global__ void separable_projection_kernel(int D, int n0, int n1, int n2, int p, int Np, int M, int nmax,
                                            const int* __restrict__ modes, const double* __restrict__ coef,
                                            const double* __restrict__ T, int64_t nc, double* __restrict__ out) {
  const int64_t total = nc * Np;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = g / Np;
    const int a = (int)(g - c * Np);
    const int i0 = (int)(c % n0);
    const int i1 = (int)((c / n0) % n1);
    const int i2 = (int)(c / ((int64_t)n0 * n1));
    const int idx[3] = {i0, i1, i2};
    double s = 0.0;
    for (int m = 0; m < M; ++m) {
      double t = coef[m];
      for (int d = 0; d < D; ++d)
        t *= T[((int64_t)(m * D + d) * nmax + idx[d]) * (p + 1) + modes[a * 3 + d]];
      s += t;
    }
    out[g] = s;
  }
  (void)n2;
}

}  // namespace

void project_separable(int D, const int32_t* shape, int p, int M, const double* coef, const double* tables,
                       double* out_device, cudaStream_t st) {
  require(D >= 1 && D <= 3, "D must be 1, 2 or 3");
  require(p >= 0 && M >= 0, "p and the term count must be >= 0");
  int n[3] = {1, 1, 1};
  int64_t nc = 1;
  int nmax = 1;
  for (int d = 0; d < D; ++d) {
    require(shape[d] >= 1, "every grid extent must be >= 1");
    n[d] = shape[d];
    nc *= shape[d];
    nmax = std::max(nmax, shape[d]);
  }
  const auto modes = modes_of(D, p);
  const int Np = (int)modes.size();
  std::vector<int> mflat((size_t)Np * 3);
  for (int a = 0; a < Np; ++a)
    for (int d = 0; d < 3; ++d) mflat[(size_t)a * 3 + d] = modes[a][d];
  // the caller's tables are [M][D][n_d][p + 1]; repack to a common stride nmax per direction
  std::vector<double> T((size_t)std::max(M, 1) * D * nmax * (p + 1), 0.0);
  size_t src = 0;
  for (int m = 0; m < M; ++m)
    for (int d = 0; d < D; ++d)
      for (int i = 0; i < n[d]; ++i)
        for (int j = 0; j <= p; ++j) T[(((size_t)m * D + d) * nmax + i) * (p + 1) + j] = tables[src++];
  DBuf<int> d_modes(mflat.size());
  DBuf<double> d_coef(std::max(M, 1)), d_T(T.size());
  BSGPU_CUDA(cudaMemcpy(d_modes.p, mflat.data(), mflat.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (M) BSGPU_CUDA(cudaMemcpy(d_coef.p, coef, M * 8, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(d_T.p, T.data(), T.size() * 8, cudaMemcpyHostToDevice));
  const int64_t total = nc * Np;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)num_sms() * 16));
  separable_projection_kernel<<<grid, 256, 0, st>>>(D, n[0], n[1], n[2], p, Np, M, nmax, d_modes.p, d_coef.p,
                                                   d_T.p, nc, out_device);
  BSGPU_CHECK_LAUNCH();
  BSGPU_CUDA(cudaStreamSynchronize(st));
}

}  // namespace bsgpu
