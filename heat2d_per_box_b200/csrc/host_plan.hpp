// Host half of a box-FGT plan: the step-0 precomputation of bfgt/boxfgt.f
// (cutoff level, plane-wave nodes, per-level 1D tables, interaction lists)
// plus the flattened work lists the device kernels consume.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace bfgt {

struct cplx {
  double re, im;
};

// Tree arrays of common/tree_routs_nd.f (layout documented in
// common/tree_routs_nd.f:1626-1706): laddr(2,0:nlevels), ilevel, iparent,
// nchild, ichild(4,nboxes), ncoll, coll(9,nboxes), all 1-based box ids.
struct TreeView {
  int nboxes = 0, nlevels = 0;
  int *itree = nullptr;
  const int *iptr = nullptr;
  const double *centers = nullptr;  // (2, nboxes)
  const double *boxsize = nullptr;  // (0:nlevels)
  int laddr(int c, int lev) const { return itree[c - 1 + 2 * lev]; }
  int ilevel(int b) const { return itree[iptr[1] + b - 2]; }
  int iparent(int b) const { return itree[iptr[2] + b - 2]; }
  int nchild(int b) const { return itree[iptr[3] + b - 2]; }
  int ichild(int j, int b) const { return itree[iptr[4] + 4 * (b - 1) + j - 2]; }
  int &ncoll(int b) const { return itree[iptr[5] + b - 2]; }
  int &coll(int j, int b) const { return itree[iptr[6] + 9 * (b - 1) + j - 2]; }
  double cen(int k, int b) const { return centers[(k - 1) + 2 * (b - 1)]; }
};

// One leaf handled by plane waves: its box, the offset indices of its center
// relative to its cutoff-level ancestor (in units of half its own box size),
// and its level.
struct PwLeaf {
  int box;  // 0-based
  int ox, oy;
  int level;
};

// A column: the PW leaves of one cutoff ancestor and level that share the
// x-offset ox (so they differ only in oy), stored contiguously in the sorted
// PwLeaf array.
struct Column {
  int begin, end;  // into the sorted PwLeaf array
  int ox;
  int icut, level;
};

// A unit of work for one CTA: consecutive columns of one cutoff ancestor and
// level.
struct Chunk {
  int begin, end;  // into the column array
  int icut;        // cutoff box index
  int level;
};

struct HostPlan {
  // inputs
  int nd = 1, norder = 0, ipoly = 0, iperiod_in = 0, nboxes = 0, nlevels = 0, precision = 0;
  double delta = 0, eps = 0;
  // step-0 scalars (boxfgt.f:130-167, 489-549)
  int npwlevel = 0;      // boxfgt-level cutoff
  int npwlevel_int = 0;  // bfgtmain-internal cutoff
  int iperiod_int = 0;
  int nlevstart = 0, nlevend = 0;
  int npw = 0, hh = 0, nexp = 0;
  int regime = 1;  // 0: periodic Fourier (A), 1: PW + near field (B), 2: near field only (C)
  bool direct_only = false;
  double delta0 = 1.0, pmax = 0, bs0 = 1;
  int nleafbox = 0, mnlist1 = 0;
  std::vector<double> ts, ws, xq;
  // per-level tables
  std::vector<cplx> tab_poly2pw;  // (n, npw, 0:nlevels), Fortran order
  std::vector<cplx> tab_pw2pot;   // (npw, n, 0:nlevels)
  std::vector<double> tab_loc;    // (n, n, -6:6, 0:nlevels)
  // first and second derivatives of tab_loc in the target coordinate
  // (tabx_loc, tabxx_loc of mk_loctab_all, bfgt_volrouts.f:407-660); ind_loc
  // is the merged band pattern of all three
  std::vector<double> tabx_loc, tabxx_loc;
  std::vector<int> ind_loc;       // (2, n+1, -6:6, 0:nlevels)
  std::vector<cplx> wshift;       // (nexp, 9) cutoff-level mp->loc shifts
  // lists (1-based box ids as in the reference)
  std::vector<int> ifpwexp, nlist1, list1;  // list1(mnlist1, nboxes)
  std::vector<int> nlistpw, listpw;         // listpw(8, nboxes)
  // device work lists
  std::vector<int> cut_box;                  // 0-based box id per cutoff box
  std::vector<int> cut_chunk_begin;          // ncut+1 offsets into chunks
  std::vector<int> cut_pw_begin;             // ncut+1 offsets into cut_pw_src/ind
  std::vector<int> cut_pw_src, cut_pw_ind;   // source cutoff index, shift index 0..8
  std::vector<PwLeaf> leaves;                // sorted by (icut, level, ox, oy)
  std::vector<Column> columns;               // sorted by (icut, level, ox)
  std::vector<Chunk> chunks;                 // groups of columns (one CTA each)
  std::vector<cplx> phase;                   // per level: (2^d offsets, npw)
  std::vector<int64_t> phase_off;            // per level offset into phase
  std::vector<double> pw_weight;             // (hh): 1, or 1/2 on the zero frequency of odd npw
  // near field: per target leaf, entries (source box, ix, iy)
  std::vector<int> nf_target, nf_level, nf_begin;  // nf_begin has ntarget+1 entries
  std::vector<int> nf_src, nf_ix, nf_iy;
  std::vector<int> nf_elev;  // per entry: level of the 1D tables it uses (its target's level)
  // per-k2 factor the cutoff translation applies to L (hh entries; empty = 1)
  std::vector<double> kscale;
  bool adjoint = false;  // this plan applies the transpose of the transform
  // work accounting
  double flops = 0, bytes = 0, tc_flops = 0, points = 0;
  double flops_form = 0, flops_eval = 0, flops_near = 0, flops_translate = 0;
  double bytes_form = 0, bytes_eval = 0, bytes_near = 0;  // compulsory HBM bytes per stage
  double tc_flops_form = 0, tc_flops_eval = 0;           // tensor-core FLOP issued (split mode)
};

// Builds the host plan; itree's colleague arrays are recomputed in place.
// Throws std::runtime_error with a message on invalid input.
void build_host_plan(HostPlan &hp, const TreeView &t, int nd, double delta, double eps, int ipoly, int iperiod,
                     int norder, int precision);

// Host half of the transpose of the transform fwd describes (f -> pot
// becomes pot_bar -> f_bar, both on leaf boxes).  Same tree lists, leaf
// offsets, phases and cutoff shifts; the plane-wave tables are swapped and
// conjugated (values->PW becomes conj(E)^T, PW->values conj(T)^T), the
// half-spectrum weight moves into the cutoff translation, and the near-field
// tables, band patterns and pair lists are transposed.
void build_adjoint_host_plan(HostPlan &adj, const HostPlan &fwd);

// A generated tree in the reference layout (caller-side test/benchmark input).
struct TreeData {
  int nboxes = 0, nlevels = 0, norder = 0;
  std::vector<int> itree;
  int iptr[8];
  std::vector<double> centers, boxsize, fvals;
};
TreeData *tree_build(int ipoly, int iperiod, double eps, double boxlen, int norder, double eta, int ng,
                     const double *gauss, int minlev, int maxlev, bool uniform);

// Node family of a leaf: x (n), umat (values->coefficients), vmat, weights.
void leaf_nodes(int ipoly, int n, std::vector<double> &x, std::vector<double> &u, std::vector<double> &v,
                std::vector<double> &w);

}  // namespace bfgt
