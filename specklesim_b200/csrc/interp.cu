// k-space interpolation between the samplings of two truncation numbers, as a sparse
// matrix: the building block of the level-dependent-K passes.  SS with a parent K
// above the child's interpolates the child's coefficients to the parent's sampling
// (Lagrange_Interpolation_New, src/lib_sie_mlfmm.f90:268-390, called from
// src/lib_sie_tri_mlfmm_interface.f90:486-507); RR goes back down by the transpose
// (anterpolation), which keeps the far sum's quadrature exact where interpolating the
// bandwidth-K products down would not.
//
// The matrix acts on one (theta, phi) component pair: inputs [a (Qc values) | b (Qc)],
// outputs [a (Qp) | b (Qp)], Q = 2K^2 + 2 in the sampling order of build_sampling with
// the +z and -z poles last; the pole entries hold Cartesian (x, y) components.  Each
// output direction is a 2p x 2p Lagrange stencil over an extended grid:
// - theta rows run past both poles.  A pole row is the pole's Cartesian value projected
//   on theta-hat and phi-hat of the column's phi; a row past a pole is the reflection
//   through it at phi + pi, with both components negated;
// - phi columns run past 0 and 2 pi and wrap.
// Every extended cell is tracked as a linear combination of at most two inputs, built
// by the same sweeps as the reference (reflection, then wrap), so that a stencil tap
// becomes matrix entries.  The stencil base is computed in binary32 as in the
// reference ((it-1.0)/K_n*K_m with a default-real literal), and the extended phi grid as
// -2 pi + dphi k, compared against 0 and 2 pi as computed.
#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "sie_internal.h"

namespace sie {

namespace {
struct Term {
  double c;
  int src;
};
struct Cell {
  Term t[2];
  int n = 0;
};
Cell neg(const Cell& a) {
  Cell r = a;
  for (int i = 0; i < r.n; i++) r.t[i].c = -r.t[i].c;
  return r;
}
}  // namespace

int interp_csr(int p, int Kc, int Kp, bool transpose, Csr& out) {
  if (p < 1 || Kc < p + 1 || Kp < 1) return fail(SIE_ERR_ARG, "interp_csr: bad stencil or truncation number");
  std::vector<double> xc, wc, xp, wp_;
  gauss_legendre(Kc, xc, wc);
  gauss_legendre(Kp, xp, wp_);
  const int Qc = 2 * Kc * Kc + 2, Qp = 2 * Kp * Kp + 2, Nsc = 2 * Kc * Kc, Nsp = 2 * Kp * Kp;
  // extended theta (2 pi down to -pi) and phi (-2 pi up to 4 pi) nodes
  const int mph = 3 * (2 * Kc);
  const double dphi = 6 * PI / mph;
  std::vector<double> at(3 * Kc + 2), ap(mph);
  for (int j = 1; j <= Kc; j++) {
    at[j - 1] = 2 * PI - std::acos(xc[Kc - j]);
    at[j + Kc] = std::acos(xc[j - 1]);
    at[2 * Kc + 1 + j] = -std::acos(xc[Kc - j]);
  }
  at[Kc] = PI;
  at[2 * Kc + 1] = 0.0;
  for (int k = 0; k < mph; k++) ap[k] = -2 * PI + dphi * k;
  // extended grid: channel 0 theta component (a inputs), 1 phi component (b inputs)
  const int nth = Kc + 2 * p + 2, nph = 2 * Kc + 2 * p + 1, KnL = 2 * Kc;
  std::vector<Cell> g((size_t)2 * nth * nph);
  auto G = [&](int ch, int r, int c) -> Cell& { return g[((size_t)ch * nth + r) * nph + c]; };
  const int ax0 = Nsc, ay0 = Qc + Nsc, axpi = Nsc + 1, aypi = Qc + Nsc + 1;  // pole inputs
  for (int c = 0; c < nph; c++) {
    const double ph = ap[c + KnL - p];
    const double ct = std::cos(ph), st = std::sin(ph);
    G(0, p, c) = Cell{{{-ct, axpi}, {-st, aypi}}, 2};
    G(0, Kc + p + 1, c) = Cell{{{ct, ax0}, {st, ay0}}, 2};
    G(1, p, c) = Cell{{{-st, axpi}, {ct, aypi}}, 2};
    G(1, Kc + p + 1, c) = Cell{{{-st, ax0}, {ct, ay0}}, 2};
  }
  for (int i = 0; i < Kc; i++)
    for (int j = 0; j < 2 * Kc; j++) {
      G(0, p + 1 + i, p + j) = Cell{{{1.0, i * 2 * Kc + j}, {0.0, 0}}, 1};
      G(1, p + 1 + i, p + j) = Cell{{{1.0, Qc + i * 2 * Kc + j}, {0.0, 0}}, 1};
    }
  for (int r = 0; r < nth; r++) {
    const double xt = at[r + 1 - p + Kc];
    for (int c = 0; c < nph; c++) {
      const double x = ap[c - p + KnL];
      int rs = -1, cs = -1;
      if (xt < 0.0 || xt >= PI) {
        rs = xt < 0.0 ? 2 * Kc + 2 * p + 2 - r : 2 * p - r;
        if (x < PI && x >= 0.0) cs = c + Kc;
        else if (x < 2 * PI && x >= PI) cs = c - Kc;
      }
      if (cs >= 0)
        for (int ch = 0; ch < 2; ch++) G(ch, r, c) = neg(G(ch, rs, cs));
    }
  }
  for (int r = 0; r < nth; r++)
    for (int c = 0; c < nph; c++) {
      const double x = ap[c - p + KnL];
      if (x >= 2 * PI)
        for (int ch = 0; ch < 2; ch++) G(ch, r, c) = G(ch, r, c - KnL);
      else if (x < 0)
        for (int ch = 0; ch < 2; ch++) G(ch, r, c) = G(ch, r, c + KnL);
    }
  // Lagrange weights over the extended nodes ext[karr + t - p .. karr + t + p - 1]
  auto weights = [p](double x, int t, int karr, const std::vector<double>& ext, std::vector<double>& wk) {
    const double* xx = ext.data() + karr + t - p;
    for (int j = 0; j < 2 * p; j++) {
      wk[j] = 1.0;
      for (int m = 0; m < 2 * p; m++)
        if (m != j) wk[j] = (x - xx[m]) / (xx[j] - xx[m]) * wk[j];
    }
  };
  // rows of the interpolation matrix (output -> {input: coefficient})
  std::vector<std::map<int, double>> rows((size_t)2 * Qp);
  std::vector<double> wt(2 * p), wph(2 * p);
  for (int it = 1; it <= Kp; it++) {
    const double theta = std::acos(xp[it - 1]);
    const int t = (int)std::floor(((float)it - 1.0f) / (float)Kp * (float)Kc) + 1;
    weights(theta, t, Kc, at, wt);
    for (int jp = 1; jp <= 2 * Kp; jp++) {
      const double phi = (double)((jp - 1) * 2) * PI / (2 * Kp);
      const int s = (int)std::floor(((float)jp - 1.0f) / (float)Kp * (float)Kc) + 1;
      weights(phi, s, 2 * Kc, ap, wph);
      const int o = (it - 1) * 2 * Kp + (jp - 1);
      for (int i = 0; i < 2 * p; i++)
        for (int j = 0; j < 2 * p; j++) {
          const double w = wph[j] * wt[i];
          for (int ch = 0; ch < 2; ch++) {
            const Cell& cl = G(ch, t + i, s + j);
            for (int k = 0; k < cl.n; k++) rows[(size_t)ch * Qp + o][cl.t[k].src] += w * cl.t[k].c;
          }
        }
    }
  }
  for (int k = 0; k < 2; k++) {  // the poles are carried over
    rows[Nsp + k][Nsc + k] = 1.0;
    rows[(size_t)Qp + Nsp + k][Qc + Nsc + k] = 1.0;
  }
  // CSR, or the CSR of the transpose
  out.rows = transpose ? 2 * Qc : 2 * Qp;
  out.cols = transpose ? 2 * Qp : 2 * Qc;
  out.ptr.assign(out.rows + 1, 0);
  for (size_t r = 0; r < rows.size(); r++)
    for (auto& e : rows[r]) out.ptr[(transpose ? e.first : (int)r) + 1]++;
  for (int r = 0; r < out.rows; r++) out.ptr[r + 1] += out.ptr[r];
  out.col.assign(out.ptr.back(), 0);
  out.val.assign(out.ptr.back(), 0.0);
  std::vector<int> fill(out.ptr.begin(), out.ptr.end() - 1);
  for (size_t r = 0; r < rows.size(); r++)  // rows ascending: transposed columns come sorted
    for (auto& e : rows[r]) {
      const int rr = transpose ? e.first : (int)r, cc = transpose ? (int)r : e.first;
      out.col[fill[rr]] = cc;
      out.val[fill[rr]++] = e.second;
    }
  return SIE_OK;
}

}  // namespace sie

// Internal export for the tests: two calls, the first with ptr == NULL for the sizes.
extern "C" int sie_internal_interp_csr(int p, int Kc, int Kp, int transpose, int* rows, int* nnz, int* ptr,
                                       int* col, double* val) {
  sie::Csr m;
  int r = sie::interp_csr(p, Kc, Kp, transpose != 0, m);
  if (r != SIE_OK) return r;
  if (rows) *rows = m.rows;
  if (nnz) *nnz = (int)m.val.size();
  if (ptr) {
    std::copy(m.ptr.begin(), m.ptr.end(), ptr);
    std::copy(m.col.begin(), m.col.end(), col);
    std::copy(m.val.begin(), m.val.end(), val);
  }
  return SIE_OK;
}
