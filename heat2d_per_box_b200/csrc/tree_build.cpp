// Caller-side generator of adaptive, level-restricted quad trees in the
// reference layout (common/tree_vol_coeffs_nd.f: vol_tree_build 440-680,
// vol_tree_find_box_refine 689-780, fun_err 855-940, update_rints 945-1090;
// common/polytens.f: tens_prod_get_rmask 1579-1617).  It produces the test
// and benchmark inputs of the transform; it is not on the transform's path.
//
// Refinement criterion (iptype = 2): a box is split when
//   sqrt(sum_{tail} c_ij^2) * (D/2)^eta / sqrt(#tail) > eps * rint / L
// where c_ij are the tensor Legendre/Chebyshev coefficients of the box's
// values, the tail is {(i+1)^2+(j+1)^2 >= n^2}, D the box size, L the root
// size and rint the running L2 norm of f over the current leaves.
// Level restriction: a leaf may not touch a box two or more levels finer
// (periodically when iperiod = 1); violating leaves are split until none
// remain, which is the minimal 2:1-balanced refinement.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "host_plan.hpp"

namespace bfgt {

namespace {

struct GaussSum {
  int ng;
  const double *g;  // ng x {cx, cy, w, a}
  double operator()(double x, double y) const {
    double s = 0;
    for (int i = 0; i < ng; i++) {
      double dx = x - g[4 * i], dy = y - g[4 * i + 1], w = g[4 * i + 2];
      s += g[4 * i + 3] * std::exp(-(dx * dx + dy * dy) / (w * w));
    }
    return s;
  }
};

struct Box {
  int level;
  int64_t ix, iy;  // integer position at its level
  int parent;      // index into boxes, -1 for root
  int child[4];    // -1 if none
  bool leaf() const { return child[0] < 0; }
};

struct Builder {
  int ipoly, iperiod, n;
  double boxlen;
  GaussSum f;
  std::vector<Box> boxes;
  std::vector<double> bsize;
  std::vector<double> xq, umat, vmat, wq;
  std::vector<std::unordered_map<int64_t, int>> grid;  // per level: key -> box

  static int64_t key(int64_t ix, int64_t iy) { return (ix << 32) ^ (iy & 0xffffffffLL); }

  double cx(const Box &b) const { return -boxlen / 2 + (b.ix + 0.5) * bsize[b.level]; }
  double cy(const Box &b) const { return -boxlen / 2 + (b.iy + 0.5) * bsize[b.level]; }

  void ensure_level(int l) {
    while ((int)bsize.size() <= l) bsize.push_back(boxlen / std::pow(2.0, (double)bsize.size()));
    while ((int)grid.size() <= l) grid.emplace_back();
  }

  void values(const Box &b, double *out) const {
    const double c0 = cx(b), c1 = cy(b), h = bsize[b.level] / 2;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) out[i + n * j] = f(c0 + xq[i] * h, c1 + xq[j] * h);
  }

  void split(int bi) {
    Box b = boxes[bi];
    ensure_level(b.level + 1);
    // child order of get_child_box_sign (common/pts_tree_nd.f:1418-1460): mm, pm, mp, pp
    for (int j = 0; j < 4; j++) {
      Box c;
      c.level = b.level + 1;
      c.ix = 2 * b.ix + (j & 1);
      c.iy = 2 * b.iy + (j >> 1);
      c.parent = bi;
      c.child[0] = c.child[1] = c.child[2] = c.child[3] = -1;
      int ci = (int)boxes.size();
      boxes.push_back(c);
      boxes[bi].child[j] = ci;
      grid[c.level][key(c.ix, c.iy)] = ci;
    }
  }
};

void tail_mask(int n, std::vector<double> &mask, double &rsum) {
  mask.assign((size_t)n * n, 0.0);
  rsum = 0;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++)
      if ((i + 1) * (i + 1) + (j + 1) * (j + 1) >= n * n) {
        mask[i + n * j] = 1.0;
        rsum += 1;
      }
  rsum = std::sqrt(rsum);
}

}  // namespace

TreeData *tree_build(int ipoly, int iperiod, double eps, double boxlen, int norder, double eta, int ng,
                     const double *gauss, int minlev, int maxlev, bool uniform) {
  if (norder < 2 || norder > 32) throw std::runtime_error("norder must be in [2,32]");
  if (!(boxlen > 0)) throw std::runtime_error("boxlen must be positive");
  if (maxlev <= 0 || maxlev > 30) maxlev = 30;
  Builder B;
  B.ipoly = ipoly;
  B.iperiod = iperiod;
  B.n = norder;
  B.boxlen = boxlen;
  B.f = GaussSum{ng, gauss};
  leaf_nodes(ipoly, norder, B.xq, B.umat, B.vmat, B.wq);
  const int n = norder, npb = n * n;
  B.ensure_level(0);
  Box root;
  root.level = 0;
  root.ix = root.iy = 0;
  root.parent = -1;
  root.child[0] = root.child[1] = root.child[2] = root.child[3] = -1;
  B.boxes.push_back(root);
  B.grid[0][Builder::key(0, 0)] = 0;

  std::vector<double> mask;
  double rsum;
  tail_mask(n, mask, rsum);
  // quadrature weights of the leaf grid on [-1,1]^2 (tensor product)
  std::vector<double> w2(npb);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) w2[i + n * j] = B.wq[i] * B.wq[j];
  auto box_l2sq = [&](const double *v, int level) {
    double s = 0, rsc = B.bsize[level] * B.bsize[level] / 4;
    for (int i = 0; i < npb; i++) s += v[i] * v[i] * w2[i] * rsc;
    return s;
  };
  std::vector<double> vals(npb);
  B.values(B.boxes[0], vals.data());
  double rintsq = box_l2sq(vals.data(), 0);
  std::vector<double> rintbs(1, rintsq);

  // level-by-level adaptive refinement
  for (int lev = 0; lev < maxlev; lev++) {
    std::vector<int> cur;
    for (int i = 0; i < (int)B.boxes.size(); i++)
      if (B.boxes[i].level == lev) cur.push_back(i);
    if (cur.empty()) break;
    const double rint = std::sqrt(std::max(rintsq, 0.0));
    const double thr = eps * std::sqrt(1.0 / (boxlen * boxlen)) * rint;
    const double rscale = std::pow(B.bsize[lev] / 2, eta);
    std::vector<char> refine(cur.size(), 0);
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < (int)cur.size(); t++) {
      if (uniform || lev < minlev) {
        refine[t] = 1;
        continue;
      }
      std::vector<double> v(npb), tmp(npb), c(npb);
      B.values(B.boxes[cur[t]], v.data());
      // coefficients: c = U v U^T (tensor transform, x index fastest)
      for (int j = 0; j < n; j++)
        for (int p = 0; p < n; p++) {
          double s = 0;
          for (int i = 0; i < n; i++) s += B.umat[p + n * i] * v[i + n * j];
          tmp[p + n * j] = s;
        }
      for (int q = 0; q < n; q++)
        for (int p = 0; p < n; p++) {
          double s = 0;
          for (int j = 0; j < n; j++) s += B.umat[q + n * j] * tmp[p + n * j];
          c[p + n * q] = s;
        }
      double e = 0;
      for (int i = 0; i < npb; i++) e += mask[i] * c[i] * c[i];
      e = std::sqrt(e) * rscale / rsum;
      if (e > thr) refine[t] = 1;
    }
    bool any = false;
    for (char r : refine) any = any || r;
    if (!any) break;
    if (uniform && lev >= minlev) break;
    for (size_t t = 0; t < cur.size(); t++)
      if (refine[t]) {
        rintsq -= rintbs[cur[t]];
        B.split(cur[t]);
      }
    rintbs.resize(B.boxes.size(), 0.0);
    std::vector<int> fresh;
    for (size_t t = 0; t < cur.size(); t++)
      if (refine[t])
        for (int j = 0; j < 4; j++) fresh.push_back(B.boxes[cur[t]].child[j]);
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < (int)fresh.size(); t++) {
      std::vector<double> v(npb);
      B.values(B.boxes[fresh[t]], v.data());
      rintbs[fresh[t]] = box_l2sq(v.data(), B.boxes[fresh[t]].level);
    }
    if (rintsq < 0) rintsq = 0;
    for (int c : fresh) rintsq += rintbs[c];
  }

  // 2:1 balance: a non-leaf box at level m may touch only non-leaf boxes at level m-1
  for (bool changed = true; changed;) {
    changed = false;
    std::vector<int> to_split;
    for (int bi = 0; bi < (int)B.boxes.size(); bi++) {
      const Box &p = B.boxes[bi];
      if (p.leaf() || p.level < 1) continue;
      const int m = p.level;
      const int64_t nm1 = (int64_t)1 << (m - 1);
      for (int dj = -1; dj <= 1; dj++)
        for (int di = -1; di <= 1; di++) {
          int64_t x = p.ix + di, y = p.iy + dj;
          const int64_t nm = (int64_t)1 << m;
          if (iperiod == 1) {
            x = (x + nm) % nm;
            y = (y + nm) % nm;
          } else if (x < 0 || y < 0 || x >= nm || y >= nm) {
            continue;
          }
          int64_t cxi = x >> 1, cyi = y >> 1;
          (void)nm1;
          // deepest existing box at level <= m-1 containing cell (cxi, cyi) of level m-1
          int lv = m - 1, found = -1;
          while (lv >= 0) {
            auto it = B.grid[lv].find(Builder::key(cxi, cyi));
            if (it != B.grid[lv].end()) {
              found = it->second;
              break;
            }
            cxi >>= 1;
            cyi >>= 1;
            lv--;
          }
          if (found >= 0 && B.boxes[found].leaf()) to_split.push_back(found);
        }
    }
    std::sort(to_split.begin(), to_split.end());
    to_split.erase(std::unique(to_split.begin(), to_split.end()), to_split.end());
    for (int bi : to_split)
      if (B.boxes[bi].leaf()) {
        B.split(bi);
        changed = true;
      }
  }

  // renumber level by level (stable in creation order) into the reference layout
  int nlevels = 0;
  for (const Box &b : B.boxes) nlevels = std::max(nlevels, b.level);
  const int nb = (int)B.boxes.size();
  std::vector<int> order(nb);
  for (int i = 0; i < nb; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return B.boxes[a].level < B.boxes[b].level; });
  std::vector<int> newid(nb);
  for (int i = 0; i < nb; i++) newid[order[i]] = i + 1;

  TreeData *T = new TreeData();
  T->nboxes = nb;
  T->nlevels = nlevels;
  T->norder = n;
  const int ltree = 2 * (nlevels + 1) + 17 * nb;
  T->itree.assign(ltree, 0);
  int *iptr = T->iptr;
  iptr[0] = 1;
  iptr[1] = 2 * (nlevels + 1) + 1;
  iptr[2] = iptr[1] + nb;
  iptr[3] = iptr[2] + nb;
  iptr[4] = iptr[3] + nb;
  iptr[5] = iptr[4] + 4 * nb;
  iptr[6] = iptr[5] + nb;
  iptr[7] = iptr[6] + 9 * nb;
  int *it = T->itree.data();
  for (int l = 0; l <= nlevels; l++) {
    it[2 * l] = 0;
    it[2 * l + 1] = -1;
  }
  for (int i = 0; i < nb; i++) {
    int l = B.boxes[order[i]].level;
    if (it[2 * l] == 0) it[2 * l] = i + 1;
    it[2 * l + 1] = i + 1;
  }
  T->centers.assign((size_t)2 * nb, 0.0);
  T->boxsize.assign(nlevels + 1, 0.0);
  for (int l = 0; l <= nlevels; l++) T->boxsize[l] = B.bsize[l];
  T->fvals.assign((size_t)npb * nb, 0.0);
  for (int i = 0; i < nb; i++) {
    const Box &b = B.boxes[order[i]];
    it[iptr[1] - 1 + i] = b.level;
    it[iptr[2] - 1 + i] = b.parent < 0 ? -1 : newid[b.parent];
    int nc = b.leaf() ? 0 : 4;
    it[iptr[3] - 1 + i] = nc;
    for (int j = 0; j < 4; j++) it[iptr[4] - 1 + 4 * i + j] = nc ? newid[b.child[j]] : -1;
    T->centers[2 * i] = B.cx(b);
    T->centers[2 * i + 1] = B.cy(b);
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < nb; i++) B.values(B.boxes[order[i]], &T->fvals[(size_t)npb * i]);
  // colleagues with the tree's periodicity (computecoll, common/tree_routs_nd.f:106-250)
  {
    TreeView tv;
    tv.nboxes = nb;
    tv.nlevels = nlevels;
    tv.itree = it;
    tv.iptr = iptr;
    tv.centers = T->centers.data();
    tv.boxsize = T->boxsize.data();
    const double bs0 = tv.boxsize[0];
    for (int i = 1; i <= nb; i++) {
      tv.ncoll(i) = 0;
      for (int j = 1; j <= 9; j++) tv.coll(j, i) = -1;
    }
    tv.ncoll(1) = 1;
    tv.coll(1, 1) = 1;
    for (int l = 1; l <= nlevels; l++)
      for (int b = tv.laddr(1, l); b <= tv.laddr(2, l); b++) {
        int dad = tv.iparent(b);
        for (int i = 1; i <= tv.ncoll(dad); i++) {
          int jb = tv.coll(i, dad);
          for (int j = 1; j <= 4; j++) {
            int kb = tv.ichild(j, jb);
            if (kb <= 0) continue;
            bool nbr = true;
            for (int k = 1; k <= 2 && nbr; k++) {
              double dis = std::fabs(tv.cen(k, kb) - tv.cen(k, b));
              if (iperiod == 1 && bs0 - dis < dis) dis = bs0 - dis;
              if (dis > 1.05 * tv.boxsize[l]) nbr = false;
            }
            if (nbr) {
              tv.ncoll(b) += 1;
              tv.coll(tv.ncoll(b), b) = kb;
            }
          }
        }
      }
  }
  return T;
}

}  // namespace bfgt
