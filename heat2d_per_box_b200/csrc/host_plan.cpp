// Step-0 precomputation of the box FGT (bfgt/boxfgt.f:130-703) on the host,
// and the flattened work lists for the device kernels.
//
// The 1D tables follow the reference routines term by term so that the
// near-field band patterns (ind_loc, thresholded in compute_sparse_pattern)
// come out identical to the reference's:
//   common/legeexps.f  legerts 2399-2530, legetayl 2536-2590, legeexps 141-215,
//                      legepol 522-555, legepols 597-630
//   common/chebexps.f  chebexps 12-180, chebpols 594-625
//   common/besseljs3d.f besseljs3d 5-169 (argument is real here)
//   common/fgtterms.f  fgtpwterms 72-141, get_pwnodes 151-179, get_periodic_pwnodes 189-209
//   bfgt/bfgt_volrouts.f mk_leg2pw_tables 58-143, mk_cheb2pw_tables 151-275,
//                      mk_pw2pgh_tables 339-401, mk_loctab_all 407-660, mk_loctab 920-1060,
//                      mk_legetab_recur 1095-1187, mk_chebtab_recur 1191-1294,
//                      compute_sparse_pattern 1300-1378
//   bfgt/bfgt_pwrouts.f g2d_mk_pw_translation_matrices 1415-1471, gnd_find_pwshift_ind 1848-1892
//   bfgt/bfgt_local.f  gnd_find_loctab_ind 1729-1765
//   common/tree_routs_nd.f computecoll 106-250, compute_mnlist1 493-600,
//                      gnd_compute_modified_list1 864-1050, gnd_find_pwexp_boxes 1266-1367,
//                      gnd_compute_listpw 1564-1615
#include "host_plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace bfgt {

namespace {

inline cplx mk(double re, double im) { return cplx{re, im}; }
inline cplx add(cplx a, cplx b) { return mk(a.re + b.re, a.im + b.im); }
inline cplx mul(cplx a, cplx b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline cplx conj(cplx a) { return mk(a.re, -a.im); }
inline cplx scal(cplx a, double s) { return mk(a.re * s, a.im * s); }
inline cplx expi(double x) { return mk(std::cos(x), std::sin(x)); }

// ---- orthogonal polynomial machinery -------------------------------------

void legepol(double x, int n, double &pol, double &der) {
  double pkm1, pk = 1, pkp1 = x;
  if (n < 2) {
    if (n == 0) {
      pol = 1;
      der = 0;
      return;
    }
    pol = x;
    der = 1;
    return;
  }
  for (int k = 1; k <= n - 1; k++) {
    pkm1 = pk;
    pk = pkp1;
    pkp1 = ((2 * k + 1) * x * pk - k * pkm1) / (k + 1);
  }
  pol = pkp1;
  der = n * (x * pkp1 - pk) / (x * x - 1);
}

void legetayl(double pol, double der, double x, double h, int n, int k, double &sum, double &sumder) {
  const double done = 1;
  double q0 = pol, q1 = der * h;
  double q2 = (2 * x * der - n * (n + done) * pol) / (1 - x * x);
  q2 = q2 * (h * h) / 2;
  sum = q0 + q1 + q2;
  sumder = q1 / h + q2 * 2 / h;
  if (k <= 2) return;
  double qi = q1, qip1 = q2;
  for (int i = 1; i <= k - 2; i++) {
    double d = 2 * x * ((i + 1) * (i + 1)) / h * qip1 - (n * (n + done) - i * (i + 1)) * qi;
    d = d / (i + 1) / (i + 2) * (h * h) / (1 - x * x);
    sum = sum + d;
    sumder = sumder + d * (i + 2) / h;
    qi = qip1;
    qip1 = d;
  }
}

// Gauss-Legendre nodes (ascending) and weights by Taylor-series Newton sweeps
// from the centre outwards.
void legerts(int itype, int n, std::vector<double> &ts, std::vector<double> &whts) {
  ts.assign(n + 2, 0.0);
  whts.assign(n + 2, 0.0);
  int k = 30;
  double d = 1, d2 = d + 1.0e-24;
  if (d2 != d) k = 54;
  int ifodd = n - 2 * (n / 2);
  const double done = 1, pi = std::atan(done) * 4, h = pi / (2 * n);
  int ii = 0;
  for (int i = n / 2 + 1; i <= n; i++) {
    ii++;
    ts[ii - 1] = -std::cos((2 * i - 1) * h);
  }
  double pol = 1, der = 0, x0 = 0;
  legepol(x0, n, pol, der);
  double x1 = ts[0];
  int n2 = (n + 1) / 2;
  double pol3 = pol, der3 = der;
  for (int kk = 1; kk <= n2; kk++) {
    if (ifodd == 1 && kk == 1) {
      ts[0] = x0;
      whts[0] = der;
      x0 = x1;
      x1 = ts[kk];
      pol3 = pol;
      der3 = der;
      continue;
    }
    int ifstop = 0;
    for (int i = 1; i <= 10; i++) {
      legetayl(pol3, der3, x0, x1 - x0, n, k, pol, der);
      x1 = x1 - pol / der;
      if (std::fabs(pol) < 1.0e-12) ifstop++;
      if (ifstop == 3) break;
    }
    ts[kk - 1] = x1;
    if (itype > 0) whts[kk - 1] = der;
    x0 = x1;
    x1 = ts[kk];
    pol3 = pol;
    der3 = der;
  }
  for (int i = (n + 1) / 2; i >= 1; i--) ts[i + n / 2 - 1] = ts[i - 1];
  for (int i = 1; i <= n / 2; i++) ts[i - 1] = -ts[n - i];
  ts.resize(n);
  if (itype <= 0) {
    whts.resize(n);
    return;
  }
  for (int i = (n + 1) / 2; i >= 1; i--) whts[i + n / 2 - 1] = whts[i - 1];
  for (int i = 1; i <= n / 2; i++) whts[i - 1] = whts[n - i];
  whts.resize(n);
  for (int i = 0; i < n; i++) whts[i] = 2 / (1 - ts[i] * ts[i]) / (whts[i] * whts[i]);
}

void legepols(double x, int n, double *p) {
  double pkm1, pk = 1, pkp1 = x;
  p[0] = 1;
  if (n == 0) return;
  p[1] = x;
  if (n < 2) return;
  for (int k = 1; k <= n - 1; k++) {
    pkm1 = pk;
    pk = pkp1;
    pkp1 = ((2 * k + 1) * x * pk - k * pkm1) / (k + 1);
    p[k + 1] = pkp1;
  }
}

void chebpols(double x, int n, double *p) {
  double pkm1, pk = 1, pkp1 = x;
  p[0] = 1;
  if (n == 0) return;
  p[1] = x;
  if (n < 2) return;
  for (int k = 1; k <= n - 1; k++) {
    pkm1 = pk;
    pk = pkp1;
    pkp1 = 2 * x * pk - pkm1;
    p[k + 1] = pkp1;
  }
}

#define A2(a, ld, i, j) (a)[((i) - 1) + (size_t)((j) - 1) * (ld)]

void legeexps2(int n, std::vector<double> &x, std::vector<double> &u, std::vector<double> &v,
               std::vector<double> &w) {
  legerts(1, n, x, w);
  u.assign((size_t)n * n, 0.0);
  v.assign((size_t)n * n, 0.0);
  for (int i = 1; i <= n; i++) legepols(x[i - 1], n - 1, &A2(u.data(), n, 1, i));
  for (int i = 1; i <= n; i++)
    for (int j = 1; j <= n; j++) A2(v.data(), n, i, j) = A2(u.data(), n, j, i);
  for (int i = 1; i <= n; i++) {
    double d = 1;
    d = d * (2 * i - 1) / 2;
    for (int j = 1; j <= n; j++) A2(u.data(), n, i, j) = A2(v.data(), n, j, i) * w[j - 1] * d;
  }
}

void chebexps2(int n, std::vector<double> &x, std::vector<double> &uu, std::vector<double> &vv,
               std::vector<double> &w) {
  const double done = 1;
  const double pi = std::atan(done) * 4;
  const double h = pi / (2 * n);
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  uu.assign((size_t)n * n, 0.0);
  vv.assign((size_t)n * n, 0.0);
  double *u = uu.data(), *v = vv.data();
  for (int i = 1; i <= n; i++) x[n - i] = std::cos((2 * i - 1) * h);
  for (int i = 1; i <= n; i++) {
    A2(u, n, 1, i) = 1;
    A2(u, n, 2, i) = x[i - 1];
  }
  for (int i = 1; i <= n; i++) {
    double tjm2 = 1, tjm1 = x[i - 1];
    w[i - 1] = 2;
    int ic = -1;
    for (int j = 2; j <= n - 1; j++) {
      double tj = 2 * x[i - 1] * tjm1 - tjm2;
      A2(u, n, j + 1, i) = tj;
      tjm2 = tjm1;
      tjm1 = tj;
      ic = -ic;
      if (ic < 0) continue;
      double rint = -2 * (done / (j + 1) - done / (j - 1));
      w[i - 1] = w[i - 1] - rint * tj;
    }
    w[i - 1] = w[i - 1] / n;
  }
  for (int i = 1; i <= n; i++) {
    double d = 0;
    for (int j = 1; j <= n; j++) d = d + A2(u, n, i, j) * A2(u, n, i, j);
    d = done / std::sqrt(d);
    for (int j = 1; j <= n; j++) A2(u, n, i, j) = A2(u, n, i, j) * d;
  }
  double ddd = std::sqrt(2.0);
  double dd = n;
  dd = done / std::sqrt(dd / 2);
  for (int i = 1; i <= n; i++) {
    for (int j = 1; j <= n; j++) A2(u, n, j, i) = A2(u, n, j, i) * dd;
    A2(u, n, 1, i) = A2(u, n, 1, i) / ddd;
  }
  dd = n;
  dd = dd / 2;
  for (int i = 1; i <= n; i++)
    for (int j = 1; j <= n; j++) A2(v, n, j, i) = A2(u, n, i, j) * dd;
  for (int i = 1; i <= n; i++)
    for (int j = 1; j <= n; j++) {
      double d = A2(v, n, j, i);
      A2(v, n, j, i) = A2(u, n, j, i) * n / 2;
      A2(u, n, j, i) = d / n * 2;
    }
  for (int i = 1; i <= n; i++) A2(v, n, 1, i) = A2(v, n, 1, i) * 2;
  for (int i = 1; i <= n; i++)
    for (int j = 1; j <= i - 1; j++) {
      std::swap(A2(u, n, j, i), A2(u, n, i, j));
      std::swap(A2(v, n, j, i), A2(v, n, i, j));
    }
}

// Miller backward recurrence for j_0..j_nterms at a real argument.
void besseljs(int nterms, double z, std::vector<double> &fjs) {
  const double upbound2 = 1.0e+40, upbound2inv = 1.0e-40, tiny = 1.0e-200, done = 1.0;
  fjs.assign(nterms + 1, 0.0);
  if (std::fabs(z) < tiny) {
    fjs[0] = done;
    return;
  }
  const double zinv = done / z;
  double fjm1 = 0, fj0 = done;
  int lwfjs = nterms + 100000, ntop = lwfjs;
  for (int i = nterms; i <= lwfjs; i++) {
    double fj1 = (2 * i + done) * zinv * fj0 - fjm1;
    if (fj1 * fj1 > upbound2) {
      ntop = i + 1;
      break;
    }
    fjm1 = fj0;
    fj0 = fj1;
  }
  std::vector<int> iscale(ntop + 1, 0);
  std::vector<double> f(ntop + 1, 0.0);
  f[ntop] = 0;
  f[ntop - 1] = done;
  for (int i = ntop - 1; i >= 1; i--) {
    f[i - 1] = (2 * i + done) * zinv * f[i] - f[i + 1];
    if (f[i - 1] * f[i - 1] > upbound2) {
      f[i] = f[i] * upbound2inv;
      f[i - 1] = f[i - 1] * upbound2inv;
      iscale[i] = 1;
    }
  }
  double sctot = 1.0;
  for (int i = 1; i <= ntop; i++) {
    sctot = sctot * done;
    if (iscale[i - 1] == 1) sctot = sctot * upbound2inv;
    f[i] = f[i] * sctot;
  }
  double g0 = std::sin(z) * zinv;
  double g1 = g0 * zinv - std::cos(z) * zinv;
  double zscale = (std::fabs(g1) > std::fabs(g0)) ? g1 / (f[1] * 1.0) : g0 / f[0];
  for (int i = 0; i <= nterms; i++) fjs[i] = f[i] * zscale;
}

// value d times (-i)^m, i.e. d / i^m
inline cplx div_ipow(double d, int m) {
  switch (m & 3) {
    case 0: return mk(d, 0);
    case 1: return mk(0, -d);
    case 2: return mk(-d, 0);
    default: return mk(0, d);
  }
}

void fgtpwterms(double bsize, double delta, double eps, int iperiod, double &pmax, int &npw) {
  const double pi = 4.0 * std::atan(1.0);
  if (iperiod == 0) {
    double rmax = bsize / std::sqrt(delta);
    double d = std::sqrt(std::log(1.0 / eps));
    pmax = 2.0 * d;
    double h = 2 * pi / (rmax + d);
    npw = 2 * ((int)(pmax / h) + 1);
  } else {
    npw = 2 * ((int)(bsize * std::sqrt(std::log(1.0 / eps) / delta) / pi) + 1) + 1;
  }
}

// ---- 1D tables -------------------------------------------------------------

// tab(n, npw): values -> PW coefficients for the leaf node family.
void mk_poly2pw(int ipoly, int n, int npw, const std::vector<double> &ws, const std::vector<double> &ts,
                double delta, double boxdim, cplx *tab) {
  std::vector<cplx> tmp((size_t)n * npw, mk(0, 0));
  std::vector<double> fjs;
  std::vector<double> lx, lu, lv, lw;
  legeexps2(n, lx, lu, lv, lw);
  std::vector<double> conv;  // Chebyshev-from-Legendre coefficients v(k,i)
  if (ipoly == 1) {
    std::vector<double> chebv((size_t)n * n);
    for (int i = 1; i <= n; i++) chebpols(lx[i - 1], n - 1, &A2(chebv.data(), n, 1, i));
    conv.assign((size_t)n * n, 0.0);
    for (int j = 1; j <= n; j++)
      for (int i = 1; i <= n; i++) {
        double dd = 0;
        for (int k = 1; k <= n; k++) dd = dd + A2(lu.data(), n, j, k) * A2(chebv.data(), n, i, k);
        A2(conv.data(), n, j, i) = dd;
      }
  }
  const double fac = boxdim / (2 * std::sqrt(delta));
  for (int j = npw / 2 + 1; j <= npw; j++) {
    double dd = ws[j - 1] * boxdim;
    cplx *col = &tmp[(size_t)n * (j - 1)];
    cplx *mir = &tmp[(size_t)n * (npw - j)];
    if (std::fabs(ts[j - 1]) < 1e-12) {
      if (ipoly == 0) {
        col[0] = mk(dd, 0);
        for (int m = 2; m <= n; m++) col[m - 1] = mk(0, 0);
      } else {
        for (int m = 0; m <= n - 1; m += 2) col[m] = mk(dd / (1.0 - m * m), 0);
        for (int m = 1; m <= n - 1; m += 2) col[m] = mk(0, 0);
        if (j != npw - j + 1)
          for (int i = 0; i < n; i++) mir[i] = conj(col[i]);
      }
      continue;
    }
    besseljs(n, ts[j - 1] * fac, fjs);
    if (ipoly == 0) {
      for (int m = 1; m <= n; m++) {
        col[m - 1] = div_ipow(dd * fjs[m - 1], m - 1);
        mir[m - 1] = conj(col[m - 1]);
      }
    } else {
      std::vector<cplx> legv(n);
      for (int m = 1; m <= n; m++) legv[m - 1] = div_ipow(dd * fjs[m - 1], m - 1);
      for (int i = 1; i <= n; i++) {
        cplx cd = mk(0, 0);
        for (int k = 1; k <= n; k++) cd = add(cd, scal(legv[k - 1], A2(conv.data(), n, k, i)));
        col[i - 1] = cd;
      }
      if (j != npw - j + 1)
        for (int i = 0; i < n; i++) mir[i] = conj(col[i]);
    }
  }
  std::vector<double> x, u, v, w;
  leaf_nodes(ipoly, n, x, u, v, w);
  for (int i = 1; i <= npw; i++)
    for (int j = 1; j <= n; j++) {
      cplx cd = mk(0, 0);
      for (int k = 1; k <= n; k++) cd = add(cd, scal(tmp[(k - 1) + (size_t)n * (i - 1)], A2(u.data(), n, k, j)));
      tab[(j - 1) + (size_t)n * (i - 1)] = cd;
    }
}

// tab(npw, n) = exp(i ts(j) x_k D / (2 sqrt(delta)))
void mk_pw2pot(int n, int npw, const std::vector<double> &ts, const std::vector<double> &xs, double delta,
               double boxdim, cplx *tab) {
  const double dsq = boxdim / 2 / std::sqrt(delta);
  const int npw2 = npw / 2;
  for (int i = 1; i <= n; i++) {
    double x = xs[i - 1] * dsq;
    for (int j1 = npw2 + 1; j1 <= npw; j1++) {
      cplx e = expi(ts[j1 - 1] * x);
      tab[(j1 - 1) + (size_t)npw * (i - 1)] = e;
      tab[(npw - j1) + (size_t)npw * (i - 1)] = conj(e);
    }
  }
}

void legetab_recur(int m, double targ, double lambda, double boxdim, double *fint, double *fx, double *fxx) {
  const double sqrtpih = 0.886226925452757940959713778283913;
  double fp[100], fpp[100];
  const double lambda2 = lambda * lambda;
  const double a = (-1 - targ) / lambda, b = (1 - targ) / lambda;
  const double erfa = std::erf(a), erfb = std::erf(b);
  const double expa = std::exp(-a * a), expb = std::exp(-b * b);
  const double d1 = lambda * (expb - expa), d2 = lambda * (expb + expa);
  fint[0] = sqrtpih * (erfb - erfa);
  fint[1] = -d1 / 2 + targ * fint[0];
  fint[2] = -d2 - targ * d1 + (lambda2 - 2.0 / 3 + 2 * (targ * targ)) * fint[0];
  fint[2] = 0.75 * fint[2];
  fint[3] = -d1 + 2 * targ * (4.0 * fint[2] / 3 - fint[0] / 3) - (0.4 - 4 * lambda2) * fint[1];
  fint[3] = 5.0 * fint[3] / 8;
  for (int k = 5; k <= m; k++) {
    int n = k - 3;
    fint[k - 1] = targ * (fint[k - 2] - fint[k - 4]) +
                  (2 * n + 1) * (lambda2 / 2 + 1.0 / ((2 * n + 3) * (2 * n - 1))) * fint[k - 3] +
                  (n - 1.0) * fint[k - 5] / (2 * n - 1);
    fint[k - 1] = (2 * n + 3.0) * fint[k - 1] / (n + 2);
  }
  fp[0] = 0;
  fp[1] = fint[0] * lambda;
  for (int k = 3; k <= m; k++) fp[k - 1] = fp[k - 3] + (2 * k - 3) * fint[k - 2] * lambda;
  fpp[0] = 0;
  fpp[1] = 0;
  for (int k = 3; k <= m; k++) fpp[k - 1] = fpp[k - 3] + (2 * k - 3) * fp[k - 2];
  int isign = 1;
  for (int k = 1; k <= m; k++) {
    double px1 = (k - 1) * k / 2.0;
    fxx[k - 1] = fpp[k - 1] - px1 * (expb + isign * expa) - 2 * (b * expb - isign * a * expa) / lambda;
    isign = -isign;
  }
  const double ww = boxdim * lambda / 2;
  for (int k = 1; k <= m; k++) {
    fint[k - 1] = fint[k - 1] * ww;
    fxx[k - 1] = fxx[k - 1] * 2 / boxdim;
  }
  for (int k = 2; k <= m; k += 2) fx[k - 1] = fp[k - 1] - d2 / lambda;
  for (int k = 1; k <= m; k += 2) fx[k - 1] = fp[k - 1] - d1 / lambda;
}

void chebtab_recur(int m, double targ, double lambda, double boxdim, double *fint, double *fx, double *fxx) {
  const double sqrtpih = 0.886226925452757940959713778283913;
  double fp[100], fpp[100];
  const double lambda2 = lambda * lambda;
  const double a = (-1 - targ) / lambda, b = (1 - targ) / lambda;
  const double erfa = std::erf(a), erfb = std::erf(b);
  const double expa = std::exp(-a * a), expb = std::exp(-b * b);
  const double d1 = lambda * (expb - expa), d2 = lambda * (expb + expa);
  fint[0] = sqrtpih * (erfb - erfa);
  fint[1] = -d1 / 2 + targ * fint[0];
  fint[2] = -d2 - targ * d1 + (lambda2 - 1 + 2 * (targ * targ)) * fint[0];
  fint[3] = -d1 + 2 * targ * fint[2] - (1 - 4 * lambda2) * fint[1];
  int isign = 1;
  for (int k = 5; k <= m; k++) {
    double dc = (isign == 1) ? d2 : d1;
    int n = k - 1;
    double dd = (n - 1.0) / (n - 3);
    fint[k - 1] = 2 * targ * fint[k - 2] + 2 * ((n - 1) * lambda2 + 1.0 / (n - 3)) * fint[k - 3] +
                  dd * (fint[k - 5] - 2 * targ * fint[k - 4]) - (1 - dd) * dc;
    isign = -isign;
  }
  fp[0] = 0;
  fp[1] = fint[0] * lambda;
  fp[2] = 4 * fint[1] * lambda;
  for (int k = 4; k <= m; k++) fp[k - 1] = (fp[k - 3] / (k - 3) + 2 * fint[k - 2] * lambda) * (k - 1);
  fpp[0] = 0;
  fpp[1] = 0;
  fpp[2] = 4 * fint[0] * lambda;
  for (int k = 4; k <= m; k++) fpp[k - 1] = (fpp[k - 3] / (k - 3) + 2 * fp[k - 2]) * (k - 1);
  isign = 1;
  for (int k = 1; k <= m; k++) {
    double tp1 = (double)((k - 1) * (k - 1));
    fxx[k - 1] = fpp[k - 1] - tp1 * (expb + isign * expa) - 2 * (b * expb - isign * a * expa) / lambda;
    isign = -isign;
  }
  const double ww = boxdim * lambda / 2;
  const double sc = 2 / boxdim;
  for (int k = 1; k <= m; k++) {
    fint[k - 1] = fint[k - 1] * ww;
    fxx[k - 1] = fxx[k - 1] * sc;
  }
  for (int k = 2; k <= m; k += 2) fx[k - 1] = fp[k - 1] - d2 / lambda;
  for (int k = 1; k <= m; k += 2) fx[k - 1] = fp[k - 1] - d1 / lambda;
}

struct LocTabCtx {
  int ipoly, n, nquad;
  std::vector<double> tnodes, umat, xnodes, wts, polyv;  // polyv(nquad, n)
};

void mk_loctab(const LocTabCtx &c, double delta, double tboxdim, double tboxcen, double scale, double *tab,
               double *tabx, double *tabxx) {
  const int n = c.n, nq = c.nquad;
  double fint[100], fx[100], fxx[100];
  std::vector<double> targs(n);
  for (int i = 0; i < n; i++) targs[i] = c.tnodes[i] / scale + tboxcen;
  const double bs = tboxdim * scale;
  const double sigma = 4 * delta / (bs * bs);
  const double lambda = std::sqrt(sigma);
  const double dmax = std::sqrt(std::log(1 / 1e-16) * sigma);
  auto zero_col = [&](int j) {
    for (int m = 1; m <= n; m++) A2(tab, n, m, j) = A2(tabx, n, m, j) = A2(tabxx, n, m, j) = 0;
  };
  auto dist = [](double targ) {
    double dis = 0;
    if (targ < -1) dis = -1 - targ;
    if (targ > 1) dis = targ - 1;
    return dis;
  };
  if (lambda <= 0.125) {
    for (int j = 1; j <= n; j++) {
      double targ = targs[j - 1];
      if (dist(targ) > dmax) {
        zero_col(j);
        continue;
      }
      if (c.ipoly == 0) legetab_recur(n, targ, lambda, bs, fint, fx, fxx);
      else chebtab_recur(n, targ, lambda, bs, fint, fx, fxx);
      for (int m = 1; m <= n; m++) {
        A2(tab, n, m, j) = fint[m - 1];
        A2(tabx, n, m, j) = fx[m - 1];
        A2(tabxx, n, m, j) = fxx[m - 1];
      }
    }
    return;
  }
  std::vector<double> wexp((size_t)nq * n);
  for (int j = 1; j <= n; j++)
    for (int i = 1; i <= nq; i++) {
      double dx = targs[j - 1] - c.xnodes[i - 1];
      A2(wexp.data(), nq, i, j) = (std::fabs(dx) < dmax) ? std::exp(-dx * dx / sigma) * c.wts[i - 1] : 0.0;
    }
  const double bsh = bs / 2;
  for (int j = 1; j <= n; j++) {
    double targ = targs[j - 1];
    if (dist(targ) > dmax) {
      zero_col(j);
      continue;
    }
    for (int m = 1; m <= n; m++) {
      double rsum = 0, rsumx = 0, rsumxx = 0;
      for (int i = 1; i <= nq; i++) {
        double dx = targ - c.xnodes[i - 1];
        double dd = -2 * dx / sigma * 2 / bs;
        double pw = A2(c.polyv.data(), nq, i, m) * A2(wexp.data(), nq, i, j);
        rsum = rsum + pw;
        rsumx = rsumx + pw * dd;
        rsumxx = rsumxx + pw * (dd * dd - 2 / delta);
      }
      A2(tab, n, m, j) = rsum * bsh;
      A2(tabx, n, m, j) = rsumx * bsh;
      A2(tabxx, n, m, j) = rsumxx * bsh;
    }
  }
}

void sparse_pattern(double eps, int n, const double *a, int *indc) {
  for (int i = 0; i <= n; i++) {
    indc[2 * i] = 0;
    indc[2 * i + 1] = -1;
  }
  double dmax = 0;
  for (int i = 0; i < n * n; i++) dmax = std::max(dmax, std::fabs(a[i]));
  if (dmax <= 2e-16) return;
  const double thr = eps * dmax / n;
  for (int i = 1; i <= n; i++)
    for (int j = 1; j <= n; j++)
      if (std::fabs(A2(a, n, j, i)) > thr) {
        indc[2 * (i - 1)] = j;
        break;
      }
  for (int i = 1; i <= n; i++)
    for (int j = n; j >= 1; j--)
      if (std::fabs(A2(a, n, j, i)) > thr) {
        indc[2 * (i - 1) + 1] = j;
        break;
      }
  for (int i = 1; i <= n; i++)
    if (indc[2 * (i - 1)] > 0) {
      indc[2 * n] = i;
      break;
    }
  for (int i = n; i >= 1; i--)
    if (indc[2 * (i - 1) + 1] > 0) {
      indc[2 * n + 1] = i;
      break;
    }
}

// tab_loc(n,n,-6:6) and ind_loc(2,n+1,-6:6) of one target level (mrefinelev = 0)
void mk_loctab_level(const LocTabCtx &c, double eps, double delta, double boxdim, double *tab_loc, double *tabx_out,
                     double *tabxx_out, int *ind_loc) {
  const int n = c.n, nl = 6;
  auto T = [&](double *base, int m, int j, int k) -> double & {
    return base[(m - 1) + (size_t)n * ((j - 1) + (size_t)n * (k + nl))];
  };
  std::vector<double> tabx_loc((size_t)n * n * 13, 0.0), tabxx_loc((size_t)n * n * 13, 0.0);
  std::vector<double> tab(n * n), tabx(n * n), tabxx(n * n);
  std::vector<int> ind(2 * (n + 1)), indx(2 * (n + 1)), indxx(2 * (n + 1));
  auto merge = [&](int k) {
    for (int j = 1; j <= n + 1; j++) {
      int i2 = std::max(ind[2 * (j - 1) + 1], std::max(indx[2 * (j - 1) + 1], indxx[2 * (j - 1) + 1]));
      int i1 = ind[2 * (j - 1)];
      if (indx[2 * (j - 1)] != 0 && i1 > indx[2 * (j - 1)]) i1 = indx[2 * (j - 1)];
      if (indxx[2 * (j - 1)] != 0 && i1 > indxx[2 * (j - 1)]) i1 = indxx[2 * (j - 1)];
      if (i2 > 0 && i1 == 0) i1 = 1;
      ind_loc[2 * ((j - 1) + (size_t)(n + 1) * (k + nl))] = i1;
      ind_loc[2 * ((j - 1) + (size_t)(n + 1) * (k + nl)) + 1] = i2;
    }
  };
  // table offsets k and their geometry (mk_loctab_all loop, m0 = 1)
  // offsets +-5 are never built (mrefinelev = 0); they get the pattern of a
  // zero table, so a request for them (a periodic level-1 image beyond the
  // cutoff, boxfgt.f:1040-1052) adds nothing
  for (int kk = -5; kk <= 5; kk += 10)
    for (int j = 1; j <= n + 1; j++) {
      ind_loc[2 * ((j - 1) + (size_t)(n + 1) * (kk + nl))] = 0;
      ind_loc[2 * ((j - 1) + (size_t)(n + 1) * (kk + nl)) + 1] = -1;
    }
  static const int ks[6] = {-1, -3, 0, -4, -2, -6};
  static const double scales[6] = {2.0, 2.0, 1.0, 1.0, 0.5, 0.5};
  for (int t = 0; t < 6; t++) {
    const int k = ks[t];
    mk_loctab(c, delta, boxdim, k / 2.0, scales[t], tab.data(), tabx.data(), tabxx.data());
    for (int j = 1; j <= n; j++)
      for (int i = 1; i <= n; i++) {
        double t0 = 0, t1 = 0, t2 = 0;
        for (int l = 1; l <= n; l++) {
          double ul = A2(c.umat.data(), n, l, i);
          t0 = t0 + ul * A2(tab.data(), n, l, j);
          t1 = t1 + ul * A2(tabx.data(), n, l, j);
          t2 = t2 + ul * A2(tabxx.data(), n, l, j);
        }
        T(tab_loc, i, j, k) = t0;
        T(tabx_loc.data(), i, j, k) = t1;
        T(tabxx_loc.data(), i, j, k) = t2;
      }
    for (int j = 1; j <= n; j++)
      for (int m = 1; m <= n; m++) {
        T(tab_loc, m, j, -k) = T(tab_loc, n - m + 1, n - j + 1, k);
        T(tabx_loc.data(), m, j, -k) = -T(tabx_loc.data(), n - m + 1, n - j + 1, k);
        T(tabxx_loc.data(), m, j, -k) = T(tabxx_loc.data(), n - m + 1, n - j + 1, k);
      }
    for (int kk : {-k, k}) {
      sparse_pattern(eps, n, &T(tab_loc, 1, 1, kk), ind.data());
      sparse_pattern(eps, n, &T(tabx_loc.data(), 1, 1, kk), indx.data());
      sparse_pattern(eps, n, &T(tabxx_loc.data(), 1, 1, kk), indxx.data());
      merge(kk);
    }
  }
  std::copy(tabx_loc.begin(), tabx_loc.end(), tabx_out);
  std::copy(tabxx_loc.begin(), tabxx_loc.end(), tabxx_out);
}

// ---- tree lists ------------------------------------------------------------

void computecoll(const TreeView &t, int nboxes0, int iperiod) {
  const double bs0 = t.boxsize[0];
  for (int i = 1; i <= nboxes0; i++) {
    t.ncoll(i) = 0;
    for (int j = 1; j <= 9; j++) t.coll(j, i) = -1;
  }
  t.ncoll(1) = 1;
  t.coll(1, 1) = 1;
  for (int ilev = 1; ilev <= t.nlevels; ilev++) {
    const double lim = 1.05 * t.boxsize[ilev];
#pragma omp parallel for schedule(static)
    for (int ibox = t.laddr(1, ilev); ibox <= t.laddr(2, ilev); ibox++) {
      int dad = t.iparent(ibox);
      for (int i = 1; i <= t.ncoll(dad); i++) {
        int jbox = t.coll(i, dad);
        for (int j = 1; j <= 4; j++) {
          int kbox = t.ichild(j, jbox);
          if (kbox <= 0) continue;
          bool nb = true;
          for (int k = 1; k <= 2 && nb; k++) {
            double dis = std::fabs(t.cen(k, kbox) - t.cen(k, ibox));
            if (iperiod == 1 && bs0 - dis < dis) dis = bs0 - dis;
            if (dis > lim) nb = false;
          }
          if (nb) {
            t.ncoll(ibox) += 1;
            t.coll(t.ncoll(ibox), ibox) = kbox;
          }
        }
      }
    }
  }
}

inline double pdist(const TreeView &t, int k, int a, int b, int iperiod) {
  double dis = std::fabs(t.cen(k, a) - t.cen(k, b));
  if (iperiod == 1) {
    double dp1 = t.boxsize[0] - dis;
    if (dp1 < dis) dis = dp1;
  }
  return dis;
}

}  // namespace

void leaf_nodes(int ipoly, int n, std::vector<double> &x, std::vector<double> &u, std::vector<double> &v,
                std::vector<double> &w) {
  if (ipoly == 0) legeexps2(n, x, u, v, w);
  else chebexps2(n, x, u, v, w);
}

namespace {

// FLOP of the near-field pass: a banded x then y contraction per pair entry
double near_flops(const HostPlan &hp) {
  const int n = hp.norder;
  const double nn = n;
  double f = 0;
  for (size_t e = 0; e < hp.nf_src.size(); e++) {
    const int *il = &hp.ind_loc[(size_t)2 * (n + 1) * 13 * hp.nf_elev[e]];
    auto band = [&](int k) {
      const int *p = il + (size_t)2 * (n + 1) * (k + 6);
      int nk = p[2 * n + 1] - p[2 * n] + 1;
      return nk < 0 ? 0 : nk;
    };
    const double nx = band(hp.nf_ix[e]), ny = band(hp.nf_iy[e]);
    if (nx == 0 || ny == 0) continue;
    f += hp.nd * 2.0 * (nx * nn * nn + nx * ny * nn);
  }
  return f;
}

}  // namespace

void build_host_plan(HostPlan &hp, const TreeView &t, int nd, double delta, double eps, int ipoly, int iperiod,
                     int norder, int precision) {
  if (nd < 1) throw std::runtime_error("nd must be >= 1");
  if (norder < 4 || norder > 32) throw std::runtime_error("norder must be in [4,32]");
  if (ipoly != 0 && ipoly != 1) throw std::runtime_error("ipoly must be 0 (Legendre) or 1 (Chebyshev)");
  if (iperiod != 0 && iperiod != 1) throw std::runtime_error("iperiod must be 0 or 1");
  if (!(delta > 0) || !(eps > 0) || !(eps < 1)) throw std::runtime_error("delta must be > 0 and 0 < eps < 1");
  const int nlevels = t.nlevels, nboxes = t.nboxes, n = norder;
  if (nlevels < 0 || nlevels > 60 || nboxes < 1) throw std::runtime_error("invalid nlevels/nboxes");
  // validate the tree arrays before they are used as indices
  if (t.laddr(1, 0) != 1 || t.laddr(2, 0) != 1) throw std::runtime_error("laddr(:,0) must be (1,1)");
  for (int l = 1; l <= nlevels; l++)
    if (t.laddr(1, l) != t.laddr(2, l - 1) + 1 || t.laddr(2, l) < t.laddr(1, l) - 1)
      throw std::runtime_error("laddr is not contiguous by level");
  const int nboxes0 = t.laddr(2, nlevels);
  if (nboxes0 > nboxes) throw std::runtime_error("laddr(2,nlevels) exceeds nboxes");
  for (int l = 0; l <= nlevels; l++)
    for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++) {
      if (t.ilevel(b) != l) throw std::runtime_error("ilevel inconsistent with laddr");
      int nc = t.nchild(b);
      if (nc != 0 && nc != 4) throw std::runtime_error("nchild must be 0 or 4");
      if (nc == 4 && l == nlevels) throw std::runtime_error("box at the finest level has children");
      for (int j = 1; j <= nc; j++) {
        int c = t.ichild(j, b);
        if (c < t.laddr(1, l + 1) || c > t.laddr(2, l + 1) || t.iparent(c) != b)
          throw std::runtime_error("ichild/iparent inconsistent");
      }
      if (l > 0) {
        int p = t.iparent(b);
        if (p < t.laddr(1, l - 1) || p > t.laddr(2, l - 1)) throw std::runtime_error("iparent out of range");
      }
    }

  hp = HostPlan();
  hp.nd = nd;
  hp.norder = n;
  hp.ipoly = ipoly;
  hp.iperiod_in = iperiod;
  hp.nboxes = nboxes;
  hp.nlevels = nlevels;
  hp.precision = precision;
  hp.delta = delta;
  hp.eps = eps;
  hp.bs0 = t.boxsize[0];

  // ---- cutoff level and number of plane waves (boxfgt.f:133-167)
  const double dcutoff = std::sqrt(delta * std::log(1.0 / eps));
  int npwlevel = nlevels + 1;
  for (int i = nlevels; i >= 0; i--)
    if (t.boxsize[i] >= dcutoff) {
      npwlevel = i;
      break;
    }
  if (t.boxsize[nlevels] > dcutoff) npwlevel = nlevels + 1;
  if (t.boxsize[0] <= dcutoff) npwlevel = 0;
  if (npwlevel <= 1 && iperiod == 1) npwlevel = 0;
  int npw = 0;
  double pmax = 0;
  if (npwlevel <= nlevels) {
    if (npwlevel <= 0) fgtpwterms(t.boxsize[0], delta, eps, iperiod, pmax, npw);
    else fgtpwterms(2 * t.boxsize[npwlevel], delta, eps, 0, pmax, npw);
  }
  hp.npwlevel = npwlevel;
  hp.pmax = pmax;
  if (npw > 200) throw std::runtime_error("npw > 200 exceeds the reference's ws(200)/ts(200) capacity");

  // ---- nodes and colleagues (boxfgt.f:489-531)
  int iperiod_i = iperiod;
  double delta0 = delta;
  hp.ts.assign(npw, 0.0);
  hp.ws.assign(npw, 0.0);
  const double pi = 4.0 * std::atan(1.0);
  if (npwlevel <= 1 && iperiod == 1) {
    const int npw2 = npw / 2;
    const double h = 2 * pi / hp.bs0, w = std::sqrt(pi * delta) / hp.bs0, hw = h * std::sqrt(delta) / 2;
    for (int j = -npw2; j <= (npw - 1) / 2; j++) {
      hp.ts[j + npw2] = j * h;
      hp.ws[j + npw2] = w * std::exp(-(hw * j) * (hw * j));
    }
    iperiod_i = 0;
    npwlevel = 0;
    delta0 = 1.0;
  } else if (npw > 0) {
    const int npw2 = npw / 2;
    const double h = pmax / npw2, w = h / (2.0 * std::sqrt(pi));
    for (int j = -npw2; j <= npw2 - 1; j++) {
      double tsj = (j + 0.5) * h;
      hp.ts[j + npw2] = tsj;
      hp.ws[j + npw2] = w * std::exp(-tsj * tsj / 4);
    }
  }
  computecoll(t, nboxes0, iperiod_i);
  hp.iperiod_int = iperiod_i;
  hp.npwlevel_int = npwlevel;
  hp.delta0 = delta0;
  std::vector<double> umat, vmat, wq;
  leaf_nodes(ipoly, n, hp.xq, umat, vmat, wq);

  int nlevend = nlevels;
  if (npwlevel < nlevels) nlevend = npwlevel;
  if (npwlevel == 0 && iperiod == 1) nlevend = -1;
  hp.nlevend = nlevend;
  hp.nleafbox = 0;
  for (int l = 1; l <= nlevels; l++)
    for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++)
      if (t.nchild(b) == 0) hp.nleafbox++;

  // ---- ifpwexp (tree_routs_nd.f:1266-1367)
  hp.ifpwexp.assign(nboxes, 0);
  if (npwlevel <= 0) hp.ifpwexp[0] = 1;
  const int ncutoff = std::max(npwlevel, 0);
  if (npwlevel <= nlevels) {
    for (int b = t.laddr(1, ncutoff); b <= t.laddr(2, ncutoff); b++) {
      if (t.nchild(b) == 0) {
        for (int j = 1; j <= t.ncoll(b); j++)
          if (t.nchild(t.coll(j, b)) > 0) {
            hp.ifpwexp[b - 1] = 1;
            break;
          }
      } else {
        hp.ifpwexp[b - 1] = 1;
      }
    }
    for (int l = ncutoff + 1; l <= nlevels; l++)
      for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++) hp.ifpwexp[b - 1] = 1;
  }

  // ---- mnlist1 (tree_routs_nd.f:493-600, isep = 1)
  {
    std::vector<int> cnt(nboxes, 0);
    cnt[0] = 1;
    for (int ilev = 1; ilev <= nlevels; ilev++) {
#pragma omp parallel for schedule(static)
      for (int b = t.laddr(1, ilev); b <= t.laddr(2, ilev); b++) {
        if (t.nchild(b) != 0) continue;
        int c = 0;
        for (int i = 1; i <= t.ncoll(b); i++) {
          int jb = t.coll(i, b);
          if (t.nchild(jb) == 0) c++;
          if (t.nchild(jb) > 0) {
            double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev + 1]) / 2.0 * 1;
            for (int j = 1; j <= 4; j++) {
              int kb = t.ichild(j, jb);
              if (kb <= 0) continue;
              bool ok = true;
              for (int k = 1; k <= 2 && ok; k++)
                if (pdist(t, k, kb, b, iperiod_i) > distest) ok = false;
              if (ok) c++;
            }
          }
        }
        int dad = t.iparent(b);
        for (int i = 1; i <= t.ncoll(dad); i++) {
          int jb = t.coll(i, dad);
          if (t.nchild(jb) != 0) continue;
          double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev - 1]) / 2.0 * 1;
          bool ok = true;
          for (int k = 1; k <= 2 && ok; k++)
            if (pdist(t, k, jb, b, iperiod_i) >= distest) ok = false;
          if (ok) c++;
        }
        cnt[b - 1] = c;
      }
    }
    hp.mnlist1 = 0;
    for (int c : cnt) hp.mnlist1 = std::max(hp.mnlist1, c);
    if (hp.mnlist1 < 1) hp.mnlist1 = 1;
  }

  // ---- modified list1 (tree_routs_nd.f:864-1050)
  const int mn = hp.mnlist1;
  hp.nlist1.assign(nboxes, 0);
  hp.list1.assign((size_t)mn * nboxes, 0);
  if (t.nchild(1) == 0) {
    hp.nlist1[0] = 1;
    hp.list1[0] = 1;
  }
  {
    const int le = (npwlevel < nlevels) ? npwlevel : nlevels;
    for (int ilev = 1; ilev <= le; ilev++) {
#pragma omp parallel for schedule(static)
      for (int b = t.laddr(1, ilev); b <= t.laddr(2, ilev); b++) {
        if (t.nchild(b) != 0) continue;
        int *l1 = &hp.list1[(size_t)mn * (b - 1)];
        int &cnt = hp.nlist1[b - 1];
        for (int i = 1; i <= t.ncoll(b); i++) {
          int jb = t.coll(i, b);
          if (t.nchild(jb) == 0) {
            if (hp.ifpwexp[b - 1] != 1 || jb != b) l1[cnt++] = jb;
          } else if (ilev < npwlevel) {
            double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev + 1]) / 2.0;
            for (int j = 1; j <= 4; j++) {
              int kb = t.ichild(j, jb);
              if (t.nchild(kb) != 0) continue;
              bool ok = true;
              for (int k = 1; k <= 2 && ok; k++)
                if (pdist(t, k, kb, b, iperiod_i) >= distest) ok = false;
              if (ok) l1[cnt++] = kb;
            }
          }
        }
        int dad = t.iparent(b);
        for (int i = 1; i <= t.ncoll(dad); i++) {
          int jb = t.coll(i, dad);
          if (t.nchild(jb) != 0) continue;
          double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev - 1]) / 2.0;
          bool ok = true;
          for (int k = 1; k <= 2 && ok; k++)
            if (pdist(t, k, jb, b, iperiod_i) >= distest) ok = false;
          if (ok) l1[cnt++] = jb;
        }
      }
    }
  }

  // ---- near-field tables (boxfgt.f:619-637; mrefinelev = 0, nloctab = 6)
  {
    LocTabCtx c;
    c.ipoly = ipoly;
    c.n = n;
    c.nquad = 50;
    std::vector<double> tv, tw;
    leaf_nodes(ipoly, n, c.tnodes, c.umat, tv, tw);
    std::vector<double> qx, qw;
    legerts(1, c.nquad, qx, qw);
    c.xnodes = qx;
    c.wts = qw;
    c.polyv.assign((size_t)c.nquad * n, 0.0);
    std::vector<double> p(n + 1);
    for (int i = 1; i <= c.nquad; i++) {
      if (ipoly == 0) legepols(c.xnodes[i - 1], n - 1, p.data());
      else chebpols(c.xnodes[i - 1], n - 1, p.data());
      for (int j = 1; j <= n; j++) A2(c.polyv.data(), c.nquad, i, j) = p[j - 1];
    }
    const size_t ntl = (size_t)n * n * 13, nil = (size_t)2 * (n + 1) * 13;
    hp.tab_loc.assign(ntl * (nlevels + 1), 0.0);
    hp.tabx_loc.assign(ntl * (nlevels + 1), 0.0);
    hp.tabxx_loc.assign(ntl * (nlevels + 1), 0.0);
    hp.ind_loc.assign(nil * (nlevels + 1), 0);
#pragma omp parallel for schedule(dynamic)
    for (int l = 0; l <= nlevels; l++)
      mk_loctab_level(c, eps, delta, t.boxsize[l], &hp.tab_loc[ntl * l], &hp.tabx_loc[ntl * l],
                      &hp.tabxx_loc[ntl * l], &hp.ind_loc[nil * l]);
  }

  hp.direct_only = (npwlevel >= nlevels && npwlevel > 0);
  hp.regime = (npwlevel == 0 && iperiod == 1) ? 0 : (hp.direct_only ? 2 : 1);
  hp.nlevstart = std::max(npwlevel, 0);

  // ---- plane-wave part (boxfgt.f:643-698)
  if (!hp.direct_only) {
    hp.npw = npw;
    hp.hh = (npw + 1) / 2;
    hp.nexp = npw * hp.hh;
    const int ls = hp.nlevstart;
    hp.tab_poly2pw.assign((size_t)n * npw * (nlevels + 1), mk(0, 0));
    hp.tab_pw2pot.assign((size_t)n * npw * (nlevels + 1), mk(0, 0));
#pragma omp parallel for schedule(dynamic)
    for (int l = ls; l <= nlevels; l++) {
      mk_poly2pw(ipoly, n, npw, hp.ws, hp.ts, delta0, t.boxsize[l], &hp.tab_poly2pw[(size_t)n * npw * l]);
      mk_pw2pot(n, npw, hp.ts, hp.xq, delta0, t.boxsize[l], &hp.tab_pw2pot[(size_t)n * npw * l]);
    }
    // cutoff-level translations, nmax = 1 (g2d_mk_pw_translation_matrices)
    const double xmin = t.boxsize[ls] / std::sqrt(delta0);
    std::vector<cplx> ww((size_t)npw * 3);
    for (int j = 0; j < npw; j++) {
      cplx z = expi(hp.ts[j] * xmin);
      ww[j + npw * 1] = mk(1, 0);
      ww[j + npw * 2] = z;
      ww[j + npw * 0] = conj(z);
    }
    hp.wshift.assign((size_t)hp.nexp * 9, mk(0, 0));
    for (int k1 = -1; k1 <= 1; k1++)
      for (int k2 = -1; k2 <= 1; k2++) {
        int k = (k1 + 1) * 3 + (k2 + 1);
        for (int j1 = 0; j1 < hp.hh; j1++)
          for (int j2 = 0; j2 < npw; j2++)
            hp.wshift[(size_t)j2 + (size_t)npw * j1 + (size_t)hp.nexp * k] = mul(ww[j2 + npw * (k2 + 1)], ww[j1 + npw * (k1 + 1)]);
      }
    // listpw (gnd_compute_listpw)
    hp.nlistpw.assign(nboxes, 0);
    hp.listpw.assign((size_t)8 * nboxes, 0);
    for (int b = t.laddr(1, ls); b <= t.laddr(2, ls); b++)
      for (int i = 1; i <= t.ncoll(b); i++) {
        int jb = t.coll(i, b);
        if (jb != b && (t.nchild(jb) > 0 || t.nchild(b) > 0)) {
          hp.listpw[(size_t)8 * (b - 1) + hp.nlistpw[b - 1]] = jb;
          hp.nlistpw[b - 1]++;
        }
      }
    // cutoff boxes and their shifted sources (gnd_find_pwshift_ind, nmax = 1)
    const int ncut = t.laddr(2, ls) - t.laddr(1, ls) + 1;
    hp.cut_box.resize(ncut);
    hp.cut_pw_begin.assign(ncut + 1, 0);
    for (int ic = 0; ic < ncut; ic++) {
      int b = t.laddr(1, ls) + ic;
      hp.cut_box[ic] = b - 1;
      for (int j = 0; j < hp.nlistpw[b - 1]; j++) {
        int jb = hp.listpw[(size_t)8 * (b - 1) + j];
        int jxyz[2];
        for (int d = 1; d <= 2; d++) {
          double dx = t.cen(d, b) - t.cen(d, jb);
          int jx = (int)std::lround(dx / t.boxsize[ls]);
          if (iperiod_i == 1) {
            int jp = (int)std::lround((dx - hp.bs0) / t.boxsize[ls]);
            int jm = (int)std::lround((dx + hp.bs0) / t.boxsize[ls]);
            if (std::abs(jx) > std::abs(jp)) jx = jp;
            if (std::abs(jx) > std::abs(jm)) jx = jm;
          }
          if (jx < -1 || jx > 1) throw std::runtime_error("listpw source is not a cutoff-level neighbour");
          jxyz[d - 1] = jx + 1;
        }
        hp.cut_pw_src.push_back(jb - t.laddr(1, ls));
        hp.cut_pw_ind.push_back(jxyz[0] + 3 * jxyz[1]);
      }
      hp.cut_pw_begin[ic + 1] = (int)hp.cut_pw_src.size();
    }
    // PW leaves, their cutoff ancestors and offsets
    std::vector<int> anc(nboxes, -1);
    for (int b = t.laddr(1, ls); b <= t.laddr(2, ls); b++) anc[b - 1] = b - t.laddr(1, ls);
    for (int l = ls + 1; l <= nlevels; l++)
      for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++) anc[b - 1] = anc[t.iparent(b) - 1];
    hp.leaves.clear();
    for (int l = ls; l <= nlevels; l++) {
      const int d = l - ls;
      const double hb = t.boxsize[l] / 2;
      for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++) {
        if (!(hp.ifpwexp[b - 1] == 1 && t.nchild(b) == 0)) continue;
        const int a = t.laddr(1, ls) + anc[b - 1];
        PwLeaf lf;
        lf.box = b - 1;
        lf.level = l;
        int o[2];
        for (int k = 1; k <= 2; k++) {
          double r = ((t.cen(k, b) - t.cen(k, a)) / hb + (double)((1 << d) - 1)) / 2.0;
          o[k - 1] = (int)std::lround(r);
          if (o[k - 1] < 0 || o[k - 1] >= (1 << d) || std::fabs(r - o[k - 1]) > 1e-6)
            throw std::runtime_error("leaf centre is not inside its cutoff ancestor");
        }
        lf.ox = o[0];
        lf.oy = o[1];
        hp.leaves.push_back(lf);
      }
    }
    std::stable_sort(hp.leaves.begin(), hp.leaves.end(), [&](const PwLeaf &x, const PwLeaf &y) {
      int ax = anc[x.box], ay = anc[y.box];
      if (ax != ay) return ax < ay;
      if (x.level != y.level) return x.level < y.level;
      if (x.ox != y.ox) return x.ox < y.ox;
      return x.oy < y.oy;
    });
    // columns (same ancestor, level, ox) and chunks of columns (same ancestor
    // and level; at most kChunkCols columns and about kChunkLeaves leaves)
    const int kChunkCols = 8, kChunkLeaves = 64;
    hp.columns.clear();
    for (size_t i = 0; i < hp.leaves.size();) {
      size_t j = i;
      while (j < hp.leaves.size() && anc[hp.leaves[j].box] == anc[hp.leaves[i].box] &&
             hp.leaves[j].level == hp.leaves[i].level && hp.leaves[j].ox == hp.leaves[i].ox)
        j++;
      hp.columns.push_back(Column{(int)i, (int)j, hp.leaves[i].ox, anc[hp.leaves[i].box], hp.leaves[i].level});
      i = j;
    }
    hp.chunks.clear();
    hp.cut_chunk_begin.assign(ncut + 1, 0);
    for (size_t c = 0; c < hp.columns.size();) {
      const PwLeaf &l0 = hp.leaves[hp.columns[c].begin];
      const int ic = anc[l0.box], lv = l0.level;
      size_t e = c;
      int nleaf = 0;
      while (e < hp.columns.size()) {
        const PwLeaf &le = hp.leaves[hp.columns[e].begin];
        if (anc[le.box] != ic || le.level != lv || (int)(e - c) >= kChunkCols) break;
        const int nl = hp.columns[e].end - hp.columns[e].begin;
        if (e > c && nleaf + nl > kChunkLeaves) break;
        nleaf += nl;
        e++;
      }
      hp.chunks.push_back(Chunk{(int)c, (int)e, ic, lv});
      c = e;
    }
    {
      size_t c = 0;
      for (int ic = 0; ic < ncut; ic++) {
        hp.cut_chunk_begin[ic] = (int)c;
        while (c < hp.chunks.size() && hp.chunks[c].icut == ic) c++;
      }
      hp.cut_chunk_begin[ncut] = (int)c;
    }
    // phase tables: phase[l][o][k] = exp(i ts_k (2o+1-2^d) boxsize(l)/2 / sqrt(delta0))
    hp.phase_off.assign(nlevels + 2, 0);
    int64_t off = 0;
    for (int l = 0; l <= nlevels; l++) {
      hp.phase_off[l] = off;
      if (l >= ls) off += (int64_t)(1 << (l - ls)) * npw;
    }
    hp.phase_off[nlevels + 1] = off;
    hp.phase.assign((size_t)off, mk(0, 0));
    const double sq = std::sqrt(delta0);
    for (int l = ls; l <= nlevels; l++) {
      const int nd_ = 1 << (l - ls);
      for (int o = 0; o < nd_; o++) {
        double dx = (double)(2 * o + 1 - nd_) * (t.boxsize[l] / 2) / sq;
        for (int k = 0; k < npw; k++) hp.phase[(size_t)hp.phase_off[l] + (size_t)o * npw + k] = expi(hp.ts[k] * dx);
      }
    }
    hp.pw_weight.assign(hp.hh, 1.0);
    if (hp.hh > npw / 2) hp.pw_weight[hp.hh - 1] = 0.5;
  }

  // ---- near-field interactions, including periodic level-1 images (boxfgt.f:925-1071)
  hp.nf_target.clear();
  hp.nf_level.clear();
  hp.nf_begin.assign(1, 0);
  hp.nf_src.clear();
  hp.nf_ix.clear();
  hp.nf_iy.clear();
  hp.nf_elev.clear();
  hp.kscale.clear();
  hp.adjoint = false;
  if (!(npwlevel == 0 && iperiod_i == 0)) {
    auto loctab_ind = [&](int ip, double tx, double ty, double sx, double sy, double sbs, int *ixy) {
      double bs = sbs / 4.0;
      double dd[2] = {(tx - sx) / bs, (ty - sy) / bs};
      for (int i = 0; i < 2; i++) {
        double dx = dd[i];
        if (ip == 1) {
          double dxp1 = dx - hp.bs0 / bs, dxm1 = dx + hp.bs0 / bs;
          if (std::fabs(dx) > std::fabs(dxp1)) dx = dxp1;
          if (std::fabs(dx) > std::fabs(dxm1)) dx = dxm1;
        }
        ixy[i] = (int)dx;
        if (ixy[i] < -6 || ixy[i] > 6) throw std::runtime_error("list1 source is not adjacent to its target");
      }
    };
    for (int l = 0; l <= nlevend; l++)
      for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++) {
        int nl1 = hp.nlist1[b - 1];
        if (nl1 == 0) continue;
        for (int j = 0; j < nl1; j++) {
          int jb = hp.list1[(size_t)mn * (b - 1) + j];
          int jlev = t.ilevel(jb);
          double bs = t.boxsize[jlev];
          int ixy[2];
          auto push = [&](int *v) {
            hp.nf_src.push_back(jb - 1);
            hp.nf_ix.push_back(v[0]);
            hp.nf_iy.push_back(v[1]);
            hp.nf_elev.push_back(l);
          };
          if (iperiod_i == 1 && jlev == 1) {
            loctab_ind(0, t.cen(1, b), t.cen(2, b), t.cen(1, jb), t.cen(2, jb), bs, ixy);
            push(ixy);
            int nimage = 0, iim[2];
            double dxyz[2], ct[2][3];
            const double bsh = bs * 0.25;
            for (int i = 0; i < 2; i++) {
              dxyz[i] = t.cen(i + 1, jb) - t.cen(i + 1, b);
              iim[i] = std::fabs(dxyz[i]) > bsh ? 1 : 0;
              nimage += iim[i];
            }
            if (nimage > 0) {
              for (int i = 0; i < 2; i++) {
                if (dxyz[i] < -bsh) ct[i][0] = t.cen(i + 1, jb) + hp.bs0;
                else if (dxyz[i] > bsh) ct[i][0] = t.cen(i + 1, jb) - hp.bs0;
                else ct[i][0] = t.cen(i + 1, jb);
              }
              if (nimage == 2) {
                ct[0][1] = t.cen(1, jb);
                ct[1][1] = ct[1][0];
                ct[0][2] = ct[0][0];
                ct[1][2] = t.cen(2, jb);
              }
              for (int k = 0; k < (1 << nimage) - 1; k++) {
                loctab_ind(0, t.cen(1, b), t.cen(2, b), ct[0][k], ct[1][k], bs, ixy);
                push(ixy);
              }
            }
          } else {
            loctab_ind(iperiod_i, t.cen(1, b), t.cen(2, b), t.cen(1, jb), t.cen(2, jb), bs, ixy);
            push(ixy);
          }
        }
        hp.nf_target.push_back(b - 1);
        hp.nf_level.push_back(l);
        hp.nf_begin.push_back((int)hp.nf_src.size());
      }
  }

  // ---- algorithmic work of one transform (FP64-equivalent, every real op once)
  {
    const double nn = n;
    double fl = 0;
    const double npwd = hp.npw, hd = hp.hh;
    const double nl = (double)hp.leaves.size() * nd;
    const double ncl = (double)hp.columns.size() * nd;
    // leaf values -> y contraction per leaf, x contraction once per column
    hp.flops_form = nl * (4 * nn * nn * hd + 6 * nn * hd) + ncl * (8 * nn * hd * npwd + 6 * nn * npwd);
    // x contraction once per column, y contraction (real part) per leaf
    hp.flops_eval = ncl * (8 * nn * hd * npwd + 6 * nn * npwd) + nl * (4 * nn * nn * hd + 6 * nn * hd);
    hp.flops_translate = (double)hp.cut_pw_src.size() * nd * 8 * hp.nexp;
    hp.bytes_form = nl * nn * nn * 8;    // leaf values read
    hp.bytes_eval = nl * nn * nn * 16;   // pot read + write
    fl += hp.flops_form + hp.flops_eval + hp.flops_translate;
    hp.flops_near = near_flops(hp);
    fl += hp.flops_near;
    hp.bytes_near = (double)hp.nf_target.size() * nd * nn * nn * 16 + (double)hp.nf_src.size() * nd * nn * nn * 8;
    hp.flops = fl;
    double leafpts = 0;
    for (int l = 0; l <= nlevels; l++)
      for (int b = t.laddr(1, l); b <= t.laddr(2, l); b++)
        if (t.nchild(b) == 0) leafpts += nn * nn;
    hp.points = leafpts * nd;
    hp.bytes = hp.points * 24.0;
  }
}

void build_adjoint_host_plan(HostPlan &a, const HostPlan &f) {
  a = f;
  a.adjoint = true;
  const int n = f.norder, npw = f.npw;
  // plane waves.  Per leaf the forward map is
  //   M = sum T(m1,k1) T(m2,k2) conj(ph(k1) ph(k2)) F(m1,m2),  L = Tr(M),
  //   pot += 2 Re sum w(k2) E(k1,x1) E(k2,x2) ph(k1) ph(k2) L(k1,k2).
  // Its transpose (real inner products) is
  //   L' = 2 w(k2) sum conj(E(k1,x1)) conj(E(k2,x2)) conj(ph ph) P(x1,x2),
  //   M' = Tr^H(L') = Tr(L') (listpw is symmetric and W(-d) = conj(W(d))),
  //   G += Re sum conj(T(m1,k1)) conj(T(m2,k2)) ph ph M'(k1,k2),
  // i.e. the forward kernels with T <- conj(E)^T, E <- conj(T)^T, weight 1
  // in the evaluation, and the factor w(k2) (= 2 w / 2) applied by the
  // translation, which commutes with it (elementwise in k2).
  if (!f.direct_only) {
    const size_t per = (size_t)n * npw;
    for (int l = f.nlevstart; l <= f.nlevels; l++) {
      const cplx *T = &f.tab_poly2pw[per * l];
      const cplx *E = &f.tab_pw2pot[per * l];
      cplx *Ta = &a.tab_poly2pw[per * l];
      cplx *Ea = &a.tab_pw2pot[per * l];
      for (int k = 0; k < npw; k++)
        for (int m = 0; m < n; m++) {
          const cplx e = E[k + (size_t)npw * m], t = T[m + (size_t)n * k];
          Ta[m + (size_t)n * k] = cplx{e.re, -e.im};
          Ea[k + (size_t)npw * m] = cplx{t.re, -t.im};
        }
    }
    a.kscale = f.pw_weight;
    a.pw_weight.assign(f.hh, 1.0);
  }
  // near field: each 1D table A(j,k) (source node j -> target node k, used on
  // the band ind_loc of column k) becomes its transpose with the band of the
  // transposed nonzero pattern; entries outside the forward band are zero, so
  // the transpose is exact for the banded operator the forward pass applies
  const size_t ntl = (size_t)n * n, nil = (size_t)2 * (n + 1);
  const size_t nslot = (size_t)13 * (f.nlevels + 1);
  for (size_t sl = 0; sl < nslot; sl++) {
    const double *tb = &f.tab_loc[ntl * sl];
    const int *ib = &f.ind_loc[nil * sl];
    double *ta = &a.tab_loc[ntl * sl];
    int *ia = &a.ind_loc[nil * sl];
    std::fill(ta, ta + ntl, 0.0);
    std::vector<int> lo(n + 1, n + 1), hi(n + 1, 0);
    const int k0 = ib[2 * n], k1 = ib[2 * n + 1];
    for (int k = k0; k >= 1 && k <= k1; k++)
      for (int j = ib[2 * (k - 1)]; j >= 1 && j <= ib[2 * (k - 1) + 1]; j++) {
        ta[(k - 1) + (size_t)n * (j - 1)] = tb[(j - 1) + (size_t)n * (k - 1)];
        lo[j] = std::min(lo[j], k);
        hi[j] = std::max(hi[j], k);
      }
    int j0 = 0, j1 = -1;
    for (int j = 1; j <= n; j++) {
      if (hi[j] > 0) {
        ia[2 * (j - 1)] = lo[j];
        ia[2 * (j - 1) + 1] = hi[j];
        if (j0 == 0) j0 = j;
        j1 = j;
      } else {
        ia[2 * (j - 1)] = 0;
        ia[2 * (j - 1) + 1] = -1;
      }
    }
    ia[2 * n] = j0;
    ia[2 * n + 1] = j1;
  }
  // transposed pair lists: grouped by the forward source, in forward order
  const size_t ne = f.nf_src.size();
  std::vector<int> tgt_of(ne);
  for (size_t tg = 0; tg < f.nf_target.size(); tg++)
    for (int e = f.nf_begin[tg]; e < f.nf_begin[tg + 1]; e++) tgt_of[e] = f.nf_target[tg];
  std::vector<size_t> ord(ne);
  for (size_t e = 0; e < ne; e++) ord[e] = e;
  std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return f.nf_src[x] < f.nf_src[y]; });
  a.nf_target.clear();
  a.nf_level.clear();
  a.nf_begin.assign(1, 0);
  a.nf_src.resize(ne);
  a.nf_ix.resize(ne);
  a.nf_iy.resize(ne);
  a.nf_elev.resize(ne);
  for (size_t i = 0; i < ne; i++) {
    const size_t e = ord[i];
    if (a.nf_target.empty() || a.nf_target.back() != f.nf_src[e]) {
      if (!a.nf_target.empty()) a.nf_begin.push_back((int)i);
      a.nf_target.push_back(f.nf_src[e]);
      a.nf_level.push_back(-1);  // entries carry their own table level
    }
    a.nf_src[i] = tgt_of[e];
    a.nf_ix[i] = f.nf_ix[e];
    a.nf_iy[i] = f.nf_iy[e];
    a.nf_elev[i] = f.nf_elev[e];
  }
  if (!a.nf_target.empty()) a.nf_begin.push_back((int)ne);
  a.flops_near = near_flops(a);
}

}  // namespace bfgt
