// Split-precision plane-wave kernels on the sm_100a tensor cores (tcgen05):
// host-side plan preparation (operand tables cut into BF16 slices, chunking,
// shared-memory sizes) and the launches.  The kernels are in split_tc.cuh;
// this translation unit instantiates the floating-slice variants and
// split_fix.cu the fixed-point ones.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bfgt.h"
#include "split_kernels.cuh"
#include "split_tc_launch.cuh"

namespace bfgt {

namespace splitk {
template void launch_form<false>(int, int, size_t, cudaStream_t, const FormTcLaunch &);
template void launch_eval<false>(int, bool, bool, int, size_t, cudaStream_t, const EvalTcLaunch &);
template void set_smem_attrs<false>();
}  // namespace splitk

using namespace splitk;

namespace {

// resident form CTAs per SM (registers and TMEM of the unpacked variants), and
// the shortest step range a long chunk is cut into
constexpr int kFormCtasPerSm = 4;
constexpr int kLongChunkSteps = 32;
constexpr int kPieceCols = 4;  // columns of a group split off a short, wide group
constexpr int kMinPieceSteps = 16;
// dynamic shared memory of an eval CTA that still lets two CTAs share an SM
// (228 KB per SM, 1 KB reserved per CTA, the kernels' static variables)
constexpr int kEvalSmemTwoPerSm = 112 * 1024;
// fixed-point slices: K-terms that one accumulation may sum and stay exact in
// FP32.  A level-0 product is at most 2^14 units of 2^-14, a level-1 term (two
// products) at most 2^15 units of 2^-22; 512 terms keep both sums within the
// 2^24 units that FP32 holds exactly.
constexpr int kFixMaxTerms = 512;
// fixed-point form CTAs hold 256 TMEM columns: two per SM (their shared
// memory is padded to this so that no third CTA waits on the allocation)
constexpr size_t kFixFormSmemMin = 80 * 1024;

// ---- host-side table preparation -----------------------------------------

uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
float bf16_to_float(uint16_t b) {
  uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
void split3_host(double v, uint16_t *s) {
  s[0] = bf16_bits((float)v);
  const double r1 = v - (double)bf16_to_float(s[0]);
  s[1] = bf16_bits((float)r1);
  const double r2 = r1 - (double)bf16_to_float(s[1]);
  s[2] = bf16_bits((float)r2);
}
// x (|x| <= 1) -> S fixed-point digits as BF16 bits: slice c = d_c 2^-(7+8c),
// d_c an integer in [-128, 128] (exact in BF16); the same cut as the kernels'
// fix_digits.
void fix_digits_host(double x, int S, uint16_t *s) {
  double sc = 128.0;
  for (int c = 0; c < S; c++) {
    const double v = std::nearbyint(x * sc) / sc;
    s[c] = bf16_bits((float)v);
    x -= v;
    sc *= 256.0;
  }
}
size_t kmajor_off_host(int r, int k, int R) {
  return (size_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

template <typename T>
int upload_vec(T *&d, const std::vector<T> &v, std::string &msg) {
  d = nullptr;
  if (v.empty()) return BFGT_OK;
  if (cudaMalloc(&d, sizeof(T) * v.size()) != cudaSuccess) {
    msg = "cudaMalloc failed (split tables)";
    return BFGT_ERR_OOM;
  }
  if (cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    msg = "cudaMemcpy failed (split tables)";
    return BFGT_ERR_CUDA;
  }
  return BFGT_OK;
}

inline cplx cmulh(cplx a, cplx b) { return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

}  // namespace

namespace {

// Dynamic shared memory of the form kernel: the double-buffered A/B operand
// slices, or Y (as float2 or double2) where that is larger, and T of the level.
size_t form_smem(const SplitPlan &sp, int n, int npw, int hh, bool yfloat) {
  const int abytes = sp.S * kRows * sp.KA * 2, bbytes = sp.S * sp.NP * sp.KA * 2;
  const int ybytes_d = kRows * (hh | 1) * 16;
  const int ybytes = yfloat ? ybytes_d / 2 : ybytes_d;
  const int ubytes = ((std::max(2 * (abytes + bbytes), ybytes) + 127) / 128) * 128;
  size_t sm = 128 + ubytes + sizeof(double2) * (size_t)n * npw;
  if (sp.fixed) sm = std::max(sm, kFixFormSmemMin);
  return sm;
}

// The eval kernel's shared memory without L: operands for step groups of eb,
// E of the level and the chunk's column phases.
size_t eval_base_smem(const SplitPlan &sp, int n, int npw, int eb) {
  const int eab = sp.S * kRows * sp.KE * 2;
  const int ebb = sp.S * (16 * eb) * sp.KE * 2;
  return 128 + ((eab + 127) / 128) * 128 + ((ebb + 127) / 128) * 128 +
         sizeof(double2) * ((size_t)npw * n + (size_t)sp.cpc * npw);
}

// Step groups of eb and as many L slots as keep two CTAs per SM (up to the
// densities a pass can pack: cpc, and 3 nd for the gradient and Hessian
// views), at least one.
void set_eval_shape(SplitPlan &sp, int n, int npw, int hh, int nd, int eb) {
  const size_t lbytes = sizeof(double2) * (size_t)npw * hh;
  const size_t ebase = eval_base_smem(sp, n, npw, eb);
  const int lcap = std::min(sp.cpc, 3 * nd);
  sp.ebatch = eb;
  sp.lslots = 1;
  while (sp.lslots < lcap && ebase + (sp.lslots + 1) * lbytes <= (size_t)kEvalSmemTwoPerSm) sp.lslots++;
  sp.smem_eval = ebase + sp.lslots * lbytes;
}

}  // namespace

int split_plan_create(DevicePlan &dp, const HostPlan &hp, std::string &msg) {
  const int n = hp.norder, npw = hp.npw, hh = hp.hh, nl = hp.nlevels, ls = hp.nlevstart;
  if (n != 8 && n != 16) {
    msg = "split precision supports norder 8 and 16";
    return BFGT_ERR_CAPACITY;
  }
  if (hh > 32) {
    msg = "split precision supports npw <= 64";
    return BFGT_ERR_CAPACITY;
  }
  SplitPlan &sp = dp.split;
  // Slices from eps (the reference's accuracy contract: relative error of
  // order eps, bfgt/boxfgt.f:133, common/fgtterms.f:72-141).  Three floating
  // slices reach about 1e-6 relative L2 (the FP32 accumulation); below
  // eps = 1e-7 fixed-point slices, 8 bits each, S of them, with an error of
  // order 2^-(8S); the exact FP32 accumulators and the FP32 rounding of the
  // level >= 2 accumulator (2^-40) bound what they can reach.
  if (hp.eps >= 1e-7) {
    sp.fixed = false;
    sp.S = 3;
  } else if (hp.eps >= 1e-9) {
    sp.fixed = true;
    sp.S = 4;
  } else if (hp.eps >= 1e-11) {
    sp.fixed = true;
    sp.S = 5;
  } else {
    msg = "split precision reaches eps >= 1e-11 (fixed-point slices); use BFGT_PREC_FP64 for smaller eps";
    return BFGT_ERR_CAPACITY;
  }
  const int S = sp.S;
  sp.cpc = kRows / n;
  sp.KA = 16;
  sp.NP = ((2 * hh + 15) / 16) * 16;
  sp.KH = ((hh + 7) / 8) * 8;
  sp.KE = ((2 * sp.KH + 15) / 16) * 16;
  sp.NB = 16;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dp.device) != cudaSuccess || nsm <= 0) {
    cudaGetLastError();
    nsm = 148;
  }
  const int slots = kFormCtasPerSm * nsm;  // resident form CTAs on the GPU
  // column groups: up to cpc columns of one (icut, level)
  const std::vector<Column> &cols = hp.columns;
  std::vector<std::pair<size_t, size_t>> groups;
  for (size_t c = 0; c < cols.size();) {
    size_t e = c;
    while (e < cols.size() && cols[e].icut == cols[c].icut && cols[e].level == cols[c].level && (int)(e - c) < sp.cpc) e++;
    groups.emplace_back(c, e);
    c = e;
  }
  // A plan whose groups fill less than a quarter of the form kernel's CTA
  // slots (a small tree, or a coarse cutoff level) splits its short, wide
  // groups (at most kLongChunkSteps steps, more than kPieceCols columns) into
  // groups of kPieceCols columns: each column is still contracted once, the
  // work spreads over more SMs.  Long groups are cut into step ranges below.
  if (!groups.empty() && 4 * (int)groups.size() <= slots) {
    std::vector<std::pair<size_t, size_t>> g2;
    for (const auto &gr : groups) {
      std::vector<int> oys;
      for (size_t q = gr.first; q < gr.second; q++)
        for (int i = cols[q].begin; i < cols[q].end; i++) oys.push_back(hp.leaves[i].oy);
      std::sort(oys.begin(), oys.end());
      const int nsteps = (int)(std::unique(oys.begin(), oys.end()) - oys.begin());
      if ((int)(gr.second - gr.first) > kPieceCols && nsteps <= kLongChunkSteps) {
        for (size_t q = gr.first; q < gr.second; q += kPieceCols) g2.emplace_back(q, std::min(q + kPieceCols, gr.second));
      } else {
        g2.push_back(gr);
      }
    }
    groups.swap(g2);
  }
  // chunks (one per group) and their oy steps.  A plan with few, long
  // chunks (a coarse cutoff level: one cutoff box at delta = 1e-2 on an
  // order-16 tree gives 35 chunks of up to 256 steps) would leave most SMs
  // idle.  When the chunks fill less than a quarter of the form kernel's CTA
  // slots, chunks of more than kLongChunkSteps steps are cut into step ranges
  // of about (total steps) / (slots), at least kMinPieceSteps: each piece is a
  // chunk of the same columns.  The form kernel's x contraction and the eval
  // kernel's H are then done once per piece; the partial expansions of the
  // pieces are summed by the same reduction as those of separate chunks.
  auto make_chunks = [&](const std::vector<std::pair<size_t, size_t>> &grs, std::vector<int4> &chunks,
                         std::vector<int> &step_begin, std::vector<int> &steps) {
    step_begin.assign(1, 0);
    for (const auto &gr : grs) {
      const size_t c = gr.first, e = gr.second;
      chunks.push_back(make_int4((int)c, (int)e, cols[c].icut, cols[c].level));
      std::vector<size_t> ptr(e - c);
      for (size_t q = c; q < e; q++) ptr[q - c] = cols[q].begin;
      for (;;) {
        int oy = INT32_MAX;
        for (size_t q = c; q < e; q++)
          if (ptr[q - c] < (size_t)cols[q].end) oy = std::min(oy, hp.leaves[ptr[q - c]].oy);
        if (oy == INT32_MAX) break;
        steps.push_back(oy);
        for (int slot = 0; slot < sp.cpc; slot++) {
          size_t q = c + slot;
          if (q < e && ptr[slot] < (size_t)cols[q].end && hp.leaves[ptr[slot]].oy == oy) {
            steps.push_back(hp.leaves[ptr[slot]].box);
            ptr[slot]++;
          } else {
            steps.push_back(-1);
          }
        }
      }
      step_begin.push_back((int)(steps.size() / (1 + sp.cpc)));
    }
    const int nch = (int)chunks.size(), total = step_begin.back();
    if (nch > 0 && 4 * nch <= slots) {
      const int smax = std::max(kMinPieceSteps, (total + slots - 1) / slots);
      std::vector<int4> pc;
      std::vector<int> pb(1, 0);
      for (int c = 0; c < nch; c++) {
        const int s0 = step_begin[c], ns = step_begin[c + 1] - s0;
        const int pieces = ns > kLongChunkSteps ? (ns + smax - 1) / smax : 1, per = (ns + pieces - 1) / pieces;
        for (int q = s0; q < s0 + ns; q += per) {
          pc.push_back(chunks[c]);
          pb.push_back(std::min(q + per, s0 + ns));
        }
      }
      chunks.swap(pc);
      step_begin.swap(pb);
    }
  };
  std::vector<int4> chunks, echunks;
  std::vector<int> step_begin, steps, estep_begin, esteps;
  make_chunks(groups, chunks, step_begin, steps);
  {
    // the eval kernel's alternative: each group of two or more columns in halves
    std::vector<std::pair<size_t, size_t>> halves;
    bool any = false;
    for (const auto &gr : groups) {
      const size_t nc = gr.second - gr.first;
      if (nc >= 2) {
        const size_t mid = gr.first + (nc + 1) / 2;
        halves.emplace_back(gr.first, mid);
        halves.emplace_back(mid, gr.second);
        any = true;
      } else {
        halves.push_back(gr);
      }
    }
    if (any) make_chunks(halves, echunks, estep_begin, esteps);
  }
  // Fixed-point slices: a form CTA accumulates n K-terms per step into the
  // same TMEM rows; chunks with more than kFixMaxTerms / n steps are cut into
  // step ranges (pieces summed by the reduction like separate chunks).
  if (sp.fixed) {
    const int smax = kFixMaxTerms / n;
    std::vector<int4> pc;
    std::vector<int> pb(1, 0);
    for (size_t c = 0; c + 1 < step_begin.size(); c++) {
      const int s0 = step_begin[c], ns = step_begin[c + 1] - s0;
      const int pieces = (ns + smax - 1) / smax, per = pieces > 0 ? (ns + pieces - 1) / pieces : 0;
      if (pieces <= 1) {
        pc.push_back(chunks[c]);
        pb.push_back(s0 + ns);
        continue;
      }
      for (int q = s0; q < s0 + ns; q += per) {
        pc.push_back(chunks[c]);
        pb.push_back(std::min(q + per, s0 + ns));
      }
    }
    chunks.swap(pc);
    step_begin.swap(pb);
  }
  // per (level, offset) operand tables
  const long long tyt = (long long)S * sp.NP * sp.KA, eyt = (long long)S * sp.NB * sp.KE;
  std::vector<long long> tyoff(nl + 1, 0), eyoff(nl + 1, 0);
  long long nty = 0, ney = 0;
  for (int l = ls; l <= nl; l++) {
    const long long noff = 1LL << (l - ls);
    tyoff[l] = nty;
    eyoff[l] = ney;
    nty += noff * tyt;
    ney += noff * eyt;
  }
  std::vector<uint16_t> TyB((size_t)nty, 0), EyB((size_t)ney, 0);
  // fixed-point column scales: Ty column (re/im, k2) and Ey column k2, per
  // level; a power of two at least the column's largest modulus over every
  // offset (the phases have modulus one), so that every entry / scale <= 1
  std::vector<double> csc, esc;
  if (sp.fixed) {
    csc.assign((size_t)(nl + 1) * sp.NP, 1.0);
    esc.assign((size_t)(nl + 1) * 16, 1.0);
  }
  auto pow2_at_least = [](double m) { return m > 0 ? std::ldexp(1.0, std::ilogb(m) + 1) : 1.0; };
  auto cut = [&](double v, double scale, uint16_t *out) {
    if (!sp.fixed) {
      split3_host(v, out);
      return;
    }
    fix_digits_host(v / scale, S, out);
  };
  for (int l = ls; l <= nl; l++) {
    const long long noff = 1LL << (l - ls);
    const cplx *T = &hp.tab_poly2pw[(size_t)n * npw * l];
    const cplx *E = &hp.tab_pw2pot[(size_t)n * npw * l];
    if (sp.fixed) {
      for (int k2 = 0; k2 < hh; k2++) {
        double m = 0;
        for (int m2 = 0; m2 < n; m2++) m = std::max(m, std::hypot(T[m2 + (size_t)n * k2].re, T[m2 + (size_t)n * k2].im));
        csc[(size_t)l * sp.NP + k2] = csc[(size_t)l * sp.NP + hh + k2] = pow2_at_least(m);
      }
      for (int k2 = 0; k2 < n; k2++) {
        double m = 0;
        for (int m2 = 0; m2 < hh; m2++) {
          const cplx e = E[m2 + (size_t)npw * k2];
          m = std::max(m, std::fabs(hp.pw_weight[m2]) * std::hypot(e.re, e.im));
        }
        esc[(size_t)l * 16 + k2] = pow2_at_least(m);
      }
    }
    for (long long o = 0; o < noff; o++) {
      const cplx *ph = &hp.phase[(size_t)hp.phase_off[l] + (size_t)o * npw];
      uint16_t *ty = &TyB[(size_t)(tyoff[l] + o * tyt)];
      const size_t ts = (size_t)sp.NP * sp.KA;  // elements per slice
      for (int k2 = 0; k2 < hh; k2++)
        for (int m2 = 0; m2 < n; m2++) {
          const cplx t = cmulh(T[m2 + (size_t)n * k2], cplx{ph[k2].re, -ph[k2].im});
          const double sc = sp.fixed ? csc[(size_t)l * sp.NP + k2] : 1.0;
          uint16_t sr[kMaxSlices], si[kMaxSlices];
          cut(t.re, sc, sr);
          cut(t.im, sc, si);
          for (int c = 0; c < S; c++) {
            *(uint16_t *)((char *)(ty + c * ts) + kmajor_off_host(k2, m2, sp.NP)) = sr[c];
            *(uint16_t *)((char *)(ty + c * ts) + kmajor_off_host(hh + k2, m2, sp.NP)) = si[c];
          }
        }
      uint16_t *ey = &EyB[(size_t)(eyoff[l] + o * eyt)];
      const size_t es = (size_t)sp.NB * sp.KE;
      for (int k2 = 0; k2 < n; k2++)
        for (int m2 = 0; m2 < hh; m2++) {
          const cplx e0 = cmulh(E[m2 + (size_t)npw * k2], ph[m2]);
          const double w = hp.pw_weight[m2];
          const double sc = sp.fixed ? esc[(size_t)l * 16 + k2] : 1.0;
          uint16_t sr[kMaxSlices], si[kMaxSlices];
          cut(w * e0.re, sc, sr);
          cut(-w * e0.im, sc, si);
          for (int c = 0; c < S; c++) {
            *(uint16_t *)((char *)(ey + c * es) + kmajor_off_host(k2, m2, sp.NB)) = sr[c];
            *(uint16_t *)((char *)(ey + c * es) + kmajor_off_host(k2, sp.KH + m2, sp.NB)) = si[c];
          }
        }
    }
  }
  sp.tyb_tile = tyt;
  sp.eyb_tile = eyt;
  sp.nchunks = (int)chunks.size();
  int rc = BFGT_OK;
  auto chk = [&](int x) {
    if (rc == BFGT_OK && x != BFGT_OK) rc = x;
  };
  chk(upload_vec(sp.chunks, chunks, msg));
  chk(upload_vec(sp.step_begin, step_begin, msg));
  chk(upload_vec(sp.steps, steps, msg));
  if (!echunks.empty()) {
    chk(upload_vec(sp.echunks, echunks, msg));
    chk(upload_vec(sp.estep_begin, estep_begin, msg));
    chk(upload_vec(sp.esteps, esteps, msg));
    sp.nechunks = (int)echunks.size();
    if (dp.nd > 1) {
      std::vector<int2> items;
      for (size_t c = 0; c < echunks.size(); c++) {
        const int rpd = (echunks[c].y - echunks[c].x) * n;
        const int dpc = std::max(std::min(dp.nd, kRows / rpd), 1);
        for (int p = 0; p < (dp.nd + dpc - 1) / dpc; p++) items.push_back(make_int2((int)c, p));
      }
      chk(upload_vec(sp.eitems, items, msg));
      sp.neitems = (int)items.size();
    }
    // (tests) BFGT_SPLIT_EVAL_HALVES=1: the eval kernel starts on the halves
    const char *ev = std::getenv("BFGT_SPLIT_EVAL_HALVES");
    sp.ehalf = ev && std::atoi(ev) == 1;
  }
  chk(upload_vec(sp.TyB, TyB, msg));
  chk(upload_vec(sp.EyB, EyB, msg));
  chk(upload_vec(sp.tyb_off, tyoff, msg));
  chk(upload_vec(sp.eyb_off, eyoff, msg));
  chk(upload_vec(sp.csc, csc, msg));
  chk(upload_vec(sp.esc, esc, msg));
  std::vector<int> zero(4, 0);
  chk(upload_vec(sp.err, zero, msg));
  if (rc != BFGT_OK) return rc;
  // the reduction and the rest of the pipeline use the tensor-core chunking
  if (dp.Mpart) cudaFree(dp.Mpart);
  dp.Mpart = nullptr;
  if (cudaMalloc(&dp.Mpart, sizeof(double2) * (size_t)dp.nd * dp.nexp * std::max<size_t>(chunks.size(), 1)) != cudaSuccess) {
    msg = "cudaMalloc failed (split partial expansions)";
    return BFGT_ERR_OOM;
  }
  {
    std::vector<int> cut_of_chunk(chunks.size());
    for (size_t c = 0; c < chunks.size(); c++) cut_of_chunk[c] = chunks[c].z;
    dp.nchunks = (int)chunks.size();
    // nd > 1: one CTA per density pass of a chunk (the passes write disjoint
    // densities; a wide chunk's passes would otherwise run one after another
    // in one CTA).  The pass count is the kernels' density_pass.
    std::vector<int> arrivals;
    if (dp.nd > 1) {
      std::vector<int2> items;
      arrivals.resize(chunks.size());
      for (size_t c = 0; c < chunks.size(); c++) {
        const int rpd = (chunks[c].y - chunks[c].x) * n;
        const int dpc = std::max(std::min(dp.nd, kRows / rpd), 1);
        const int npass = (dp.nd + dpc - 1) / dpc;
        arrivals[c] = npass;
        for (int p = 0; p < npass; p++) items.push_back(make_int2((int)c, p));
      }
      chk(upload_vec(sp.items, items, msg));
      sp.nitems = (int)items.size();
      sp.items_nd = dp.nd;
    }
    chk(build_reduce_groups(dp, cut_of_chunk, msg, arrivals));
  }
  dp.nchunks = (int)chunks.size();
  // shared memory.  Y as float2 when, as double2, it would be the largest
  // user of the form kernel's area (unpacked plans with floating slices; the
  // packed kernel and fixed-point slices keep double2).  Eval: groups of ebmax
  // steps (8 floating, 4 fixed-point: three accumulators), or of half that if
  // only that keeps two CTAs per SM with one L slot.
  {
    const int abytes = S * kRows * sp.KA * 2, bbytes = S * sp.NP * sp.KA * 2;
    const int ybytes_d = kRows * (hh | 1) * 16;
    sp.yfloat = !sp.fixed && hp.nd == 1 && ybytes_d > 2 * (abytes + bbytes);
    sp.smem_form = form_smem(sp, n, npw, hh, sp.yfloat);
    const size_t lbytes = sizeof(double2) * (size_t)npw * hh;
    const int ebmax = sp.fixed ? kEvalBatchFix : kEvalBatchMax;
    int eb = ebmax;
    if (eval_base_smem(sp, n, npw, ebmax) + lbytes > (size_t)kEvalSmemTwoPerSm &&
        eval_base_smem(sp, n, npw, ebmax / 2) + lbytes <= (size_t)kEvalSmemTwoPerSm)
      eb = ebmax / 2;
    set_eval_shape(sp, n, npw, hh, hp.nd, eb);
  }
  // x-contraction tiles per form thread (npw <= 64: at most 256 tiles)
  sp.nt = ((((npw + 1) / 2) * ((hh + 3) / 4)) + kThreads - 1) / kThreads;
  if (sp.smem_form > (size_t)kMaxDynSmem || sp.smem_eval > (size_t)kMaxDynSmem) {
    msg = "split precision: shared memory need exceeds 227 KB";
    return BFGT_ERR_CAPACITY;
  }
  if (sp.fixed) set_smem_attrs<true>();
  else set_smem_attrs<false>();
  sp.wait_iters = kWaitIters;
  // tensor-core FLOP issued per transform (every slice product counted)
  const double nsteps_total = (double)(steps.size() / (1 + sp.cpc));
  const double prods = sp.fixed ? S * (S + 1) / 2.0 : 6.0;
  sp.tc_flops_form = nsteps_total * hp.nd * prods * (sp.KA / 16) * 2.0 * kRows * sp.NP * 16;
  sp.tc_flops_eval = nsteps_total * hp.nd * prods * (sp.KE / 16) * 2.0 * kRows * sp.NB * 16;
  return rc;
}

void split_plan_destroy(DevicePlan &dp) {
  SplitPlan &sp = dp.split;
  void *ptrs[] = {sp.chunks, sp.step_begin, sp.steps, sp.echunks, sp.estep_begin, sp.esteps, sp.eitems,
                  sp.TyB, sp.EyB, sp.tyb_off, sp.eyb_off, sp.err, sp.items,
                  sp.csc, sp.esc};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  sp = SplitPlan();
}

namespace {

// The plan's {chunk, pass} items if they were cut for its density count (a
// gradient or Hessian view of the eval stage has 2 nd or 3 nd densities and
// runs whole chunks), and the CTA count that goes with the choice.
const int2 *split_items(const DevicePlan &dp) {
  return dp.split.items && dp.nd == dp.split.items_nd ? dp.split.items : nullptr;
}
int split_ctas(const DevicePlan &dp) { return split_items(dp) ? dp.split.nitems : dp.split.nchunks; }
// the eval kernel's work: the chunks, or their column halves (ehalf); items
// of the halves exist for the plan's own density count, as the chunks' do
bool eval_halves(const DevicePlan &dp) { return dp.split.ehalf && dp.split.nechunks > 0; }
const int2 *eval_items(const DevicePlan &dp) {
  if (!eval_halves(dp)) return split_items(dp);
  return dp.split.eitems && dp.nd == dp.split.items_nd ? dp.split.eitems : nullptr;
}
int eval_ctas(const DevicePlan &dp) {
  if (!eval_halves(dp)) return split_ctas(dp);
  return eval_items(dp) ? dp.split.neitems : dp.split.nechunks;
}

FormTcArgs form_args(const DevicePlan &dp, long long elem_off) {
  const SplitPlan &sp = dp.split;
  return FormTcArgs{sp.chunks, sp.step_begin, sp.steps, dp.columns, sp.TyB, sp.tyb_off, sp.tyb_tile, dp.T, dp.PH,
                    dp.ph_off, dp.Mpart, reduce_args(dp), sp.err, dp.nd, dp.n, dp.npw, dp.hh, dp.nexp, sp.cpc,
                    sp.NP, sp.KA, sp.wait_iters, elem_off, split_items(dp), sp.csc, sp.S, 0};
}

EvalTcArgs eval_args(const DevicePlan &dp, long long elem_off) {
  const SplitPlan &sp = dp.split;
  const bool h = eval_halves(dp);
  return EvalTcArgs{h ? sp.echunks : sp.chunks, h ? sp.estep_begin : sp.step_begin, h ? sp.esteps : sp.steps,
                    dp.columns, sp.EyB, sp.eyb_off, sp.eyb_tile, dp.E, dp.PH, dp.ph_off, dp.L, sp.err, dp.nd, dp.n,
                    dp.npw, dp.hh, dp.nexp, sp.cpc, sp.NB, sp.KE, sp.KH, sp.lslots, sp.ebatch, sp.wait_iters,
                    elem_off, eval_items(dp), sp.esc, sp.S, 0};
}

// variant: 0, 1 = unpacked with 1, 2 x-contraction tiles per thread (+2 with
// Y as float2); 4 = packed; +5 for n = 16; +10 with fixed-point slices
constexpr int kFormVariants = 20;
int form_variant(const DevicePlan &dp) {
  return (dp.nd > 1 ? 4 : dp.split.nt - 1 + (dp.split.yfloat ? 2 : 0)) + (dp.n == 16 ? 5 : 0) +
         (dp.split.fixed ? 10 : 0);
}
void launch_form_any(int variant, int grid, size_t smem, cudaStream_t s, const FormTcLaunch &lp) {
  if (variant >= 10) launch_form<true>(variant - 10, grid, smem, s, lp);
  else launch_form<false>(variant, grid, smem, s, lp);
}

// variant = nnt (column tiles of H) + 16 pack + 32 (n = 16) + 64 fixed-point
constexpr int kEvalVariants = 128;
int eval_variant(const DevicePlan &dp) {
  return (dp.hh + 3) / 4 + 16 * (dp.nd > 1 ? 1 : 0) + 32 * (dp.n == 16 ? 1 : 0) + 64 * (dp.split.fixed ? 1 : 0);
}
void launch_eval_any(int v, int grid, size_t smem, cudaStream_t s, const EvalTcLaunch &lp) {
  if (v & 64) launch_eval<true>(v & 15, (v & 16) != 0, (v & 32) != 0, grid, smem, s, lp);
  else launch_eval<false>(v & 15, (v & 16) != 0, (v & 32) != 0, grid, smem, s, lp);
}

}  // namespace

void split_form(DevicePlan &dp, const double *d_fvals, cudaStream_t s) {
  FormTcLaunch lp{form_args(dp, 0), nullptr, nullptr, d_fvals};
  launch_form_any(form_variant(dp), split_ctas(dp), dp.split.smem_form, s, lp);
}

void split_eval(DevicePlan &dp, double *d_pot, cudaStream_t s) {
  EvalTcLaunch lp{eval_args(dp, 0), nullptr, nullptr, d_pot};
  launch_eval_any(eval_variant(dp), eval_ctas(dp), dp.split.smem_eval, s, lp);
}

int split_autotune(DevicePlan &dp, cudaStream_t s, double *report, std::string &msg) {
  for (int i = 0; i < 4; i++) report[i] = 0;
  SplitPlan &sp = dp.split;
  if (dp.precision != BFGT_PREC_SPLIT || dp.direct_only || sp.nchunks == 0) return BFGT_OK;
  const size_t elems = (size_t)dp.nd * dp.n * dp.n * dp.nboxes;
  double *f = nullptr, *p = nullptr;
  if (cudaMalloc(&f, sizeof(double) * elems) != cudaSuccess || cudaMalloc(&p, sizeof(double) * elems) != cudaSuccess) {
    cudaGetLastError();
    if (f) cudaFree(f);
    msg = "cudaMalloc failed (autotuner scratch)";
    return BFGT_ERR_OOM;
  }
  cudaMemsetAsync(f, 0, sizeof(double) * elems, s);
  cudaMemsetAsync(p, 0, sizeof(double) * elems, s);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto time_ms = [&](auto &&launch) {
    launch();  // warm-up
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; r++) launch();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / 3.0;
  };
  // form: Y staged as float2 or double2 (unpacked floating-slice plans) and
  // 1 or 2 x-contraction tiles per thread (unpacked plans; the minimum count
  // is the only choice when it is 2)
  struct FormShape {
    bool yf;
    int nt;
  };
  std::vector<FormShape> fc;
  const bool packed = dp.nd > 1;
  const int nt_min = sp.nt;
  for (int yf = 0; yf < 2; yf++)
    for (int nt = nt_min; nt <= 2; nt++) {
      if ((yf && (sp.fixed || packed)) || (packed && nt != nt_min)) continue;
      if (form_smem(sp, dp.n, dp.npw, dp.hh, yf != 0) > (size_t)kMaxDynSmem) continue;
      fc.push_back(FormShape{yf != 0, nt});
    }
  const FormShape f0{sp.yfloat, sp.nt};
  FormShape bf = f0;
  double tf = 1e30;
  for (const FormShape &c : fc) {
    sp.yfloat = c.yf;
    sp.nt = c.nt;
    sp.smem_form = form_smem(sp, dp.n, dp.npw, dp.hh, c.yf);
    const double ms = time_ms([&] { split_form(dp, f, s); });
    if (ms < tf) tf = ms, bf = c;
  }
  sp.yfloat = bf.yf;
  sp.nt = bf.nt;
  sp.smem_form = form_smem(sp, dp.n, dp.npw, dp.hh, bf.yf);
  // eval: step groups of 8, 4 or 2 (up to the slices' maximum), each with the
  // L slots that keep two CTAs per SM
  const int ebmax = sp.fixed ? kEvalBatchFix : kEvalBatchMax;
  std::vector<int> ec;
  for (int eb = ebmax; eb >= 2; eb /= 2) {
    SplitPlan t = sp;
    set_eval_shape(t, dp.n, dp.npw, dp.hh, dp.nd, eb);
    if (t.smem_eval <= (size_t)kMaxDynSmem) ec.push_back(eb);
  }
  // and, where the chunks have column halves, the halves (twice the CTAs)
  int be = sp.ebatch;
  bool bh = sp.ehalf;
  double te = 1e30;
  int ne = 0;
  for (int half = 0; half < (sp.nechunks > 0 ? 2 : 1); half++)
    for (int eb : ec) {
      sp.ehalf = half != 0;
      set_eval_shape(sp, dp.n, dp.npw, dp.hh, dp.nd, eb);
      const double ms = time_ms([&] { split_eval(dp, p, s); });
      ne++;
      if (ms < te) te = ms, be = eb, bh = sp.ehalf;
    }
  sp.ehalf = bh;
  set_eval_shape(sp, dp.n, dp.npw, dp.hh, dp.nd, be);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  cudaFree(f);
  cudaFree(p);
  if (cudaGetLastError() != cudaSuccess) {
    msg = "CUDA error while autotuning";
    return BFGT_ERR_CUDA;
  }
  if (split_check(dp) != BFGT_OK) {
    msg = "a bounded device-side wait gave up while autotuning";
    return BFGT_ERR_TIMEOUT;
  }
  report[0] = tf;
  report[1] = te;
  report[2] = (double)fc.size();
  report[3] = (double)ne;
  return BFGT_OK;
}

int split_batch_create(SplitBatch &b, const std::vector<DevicePlan *> &plans, const std::vector<long long> &offs,
                       std::string &msg) {
  split_batch_destroy(b);
  std::vector<FormTcArgs> fd;
  std::vector<EvalTcArgs> ed;
  // the plans' work items (chunks, or chunk passes), grouped by kernel
  // variant (form_variant, eval_variant); within a group the plans keep their
  // order
  std::vector<std::vector<int2>> fw(kFormVariants), ew(kEvalVariants);
  std::vector<size_t> fsm(kFormVariants, 0), esm(kEvalVariants, 0);
  for (size_t i = 0; i < plans.size(); i++) {
    DevicePlan &dp = *plans[i];
    fd.push_back(form_args(dp, offs[i]));
    ed.push_back(eval_args(dp, offs[i]));
    if (dp.precision != BFGT_PREC_SPLIT || dp.direct_only) continue;
    const int fv = form_variant(dp), ev = eval_variant(dp);
    for (int c = 0; c < split_ctas(dp); c++) fw[fv].push_back(make_int2((int)i, c));
    for (int c = 0; c < eval_ctas(dp); c++) ew[ev].push_back(make_int2((int)i, c));
    fsm[fv] = std::max(fsm[fv], dp.split.smem_form);
    esm[ev] = std::max(esm[ev], dp.split.smem_eval);
  }
  std::vector<int2> fall, eall;
  for (int v = 0; v < kFormVariants; v++)
    if (!fw[v].empty()) {
      b.form_groups.push_back(SplitBatch::Group{v, (int)fall.size(), (int)fw[v].size(), fsm[v]});
      fall.insert(fall.end(), fw[v].begin(), fw[v].end());
    }
  for (int v = 0; v < kEvalVariants; v++)
    if (!ew[v].empty()) {
      b.eval_groups.push_back(SplitBatch::Group{v, (int)eall.size(), (int)ew[v].size(), esm[v]});
      eall.insert(eall.end(), ew[v].begin(), ew[v].end());
    }
  int rc = BFGT_OK;
  auto chk = [&](int x) {
    if (rc == BFGT_OK && x != BFGT_OK) rc = x;
  };
  FormTcArgs *dfd = nullptr;
  EvalTcArgs *ded = nullptr;
  chk(upload_vec(dfd, fd, msg));
  chk(upload_vec(ded, ed, msg));
  chk(upload_vec(b.form_work, fall, msg));
  chk(upload_vec(b.eval_work, eall, msg));
  b.form_descs = dfd;
  b.eval_descs = ded;
  return rc;
}

void split_batch_form(const SplitBatch &b, const double *fbase, cudaStream_t s) {
  for (const SplitBatch::Group &g : b.form_groups) {
    FormTcLaunch lp{};
    lp.descs = static_cast<const FormTcArgs *>(b.form_descs);
    lp.work = b.form_work + g.begin;
    lp.fbase = fbase;
    launch_form_any(g.variant, g.count, g.smem, s, lp);
  }
}

void split_batch_eval(const SplitBatch &b, double *pbase, cudaStream_t s) {
  for (const SplitBatch::Group &g : b.eval_groups) {
    EvalTcLaunch lp{};
    lp.descs = static_cast<const EvalTcArgs *>(b.eval_descs);
    lp.work = b.eval_work + g.begin;
    lp.pbase = pbase;
    launch_eval_any(g.variant, g.count, g.smem, s, lp);
  }
}

int split_batch_launches(const SplitBatch &b) { return (int)(b.form_groups.size() + b.eval_groups.size()); }

void split_batch_destroy(SplitBatch &b) {
  void *ptrs[] = {b.form_descs, b.eval_descs, b.form_work, b.eval_work};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  b = SplitBatch();
}

unsigned int split_default_wait_iters() { return kWaitIters; }

int split_check(DevicePlan &dp) {
  if (!dp.split.err) return BFGT_OK;
  int h[4] = {0, 0, 0, 0};
  if (cudaMemcpy(h, dp.split.err, sizeof(int) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return BFGT_ERR_CUDA;
  if (h[0]) {
    cudaMemset(dp.split.err, 0, sizeof(int) * 4);
    return BFGT_ERR_TIMEOUT;
  }
  return BFGT_OK;
}

}  // namespace bfgt
