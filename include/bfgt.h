/*
 * bfgt.h -- C ABI of the B200 box fast Gauss transform (libbfgt_b200.so).
 *
 * The drop-in entry point is boxfgt_, the symbol gfortran emits for
 *   call boxfgt(nd,ndim,delta,eps,ipoly,iperiod,norder,npbox,nboxes,nlevels,
 *               ltree,itree,iptr,centers,boxsize,fvals,ifpgh,pot,grad,hess,
 *               ifnewtree,ntarg,targs,ifpghtarg,pote,grade,hesse,timeinfo)
 * (bfgt/boxfgt.f:5-8).  Every argument is passed by reference, integers are
 * 32-bit, reals are double, arrays are Fortran column-major, and there are no
 * hidden character-length arguments.  All arrays are host memory owned by the
 * caller, exactly as for the Fortran routine.
 *
 * The plan API (bfgt_plan_*) is the device-resident form of the same
 * transform: the tree-dependent precomputation (boxfgt.f step 0) is done once
 * and the transform runs on device pointers, on a caller-supplied stream.
 *
 * Errors: the reference routine has no error argument.  boxfgt_ keeps the void
 * signature and records failures in bfgt_last_error(); when the environment
 * variable BFGT_ABORT_ON_ERROR is set it prints the message and aborts instead
 * of returning with pot untouched.  The bfgt_* functions return one of the
 * BFGT_* status codes below.
 */
#ifndef BFGT_H
#define BFGT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define BFGT_OK 0
#define BFGT_ERR_ARG 1          /* unsupported or inconsistent argument       */
#define BFGT_ERR_TREE 2         /* tree arrays are not a valid 2:1 quad tree  */
#define BFGT_ERR_CAPACITY 3     /* npw, norder or nd beyond the built kernels */
#define BFGT_ERR_OOM 4          /* device allocation failed                  */
#define BFGT_ERR_CUDA 5         /* a CUDA runtime call failed                */
#define BFGT_ERR_NODEVICE 6     /* no CUDA device visible                     */
#define BFGT_ERR_TIMEOUT 7      /* a bounded device-side wait gave up         */

/* precision modes of a plan */
#define BFGT_PREC_FP64 0        /* every contraction in FP64                   */
#define BFGT_PREC_SPLIT 1       /* tensor-core split-FP16 slices, FP32 accum.,
                                   FP64 phases and FP64 cross-leaf accumulation */

/* Replaces bfgt/boxfgt.f:5-286 (boxfgt).  Runs in the precision set by
   bfgt_set_default_precision (FP64 unless chosen otherwise), on a cached plan
   when the tree and arguments repeat (bfgt_plan_cache_info).  Supported:
   ndim=2, ifpgh=1, 2, 3,
   ifpghtarg=0..3, ifnewtree=0 (ifpgh=1, ifpghtarg=0 is what every solver in
   the reference uses, hpots/hpots2dadap.f:79-106).  pot (and
   grad(nd,2,npbox,nboxes), hess(nd,3,npbox,nboxes) as ifpgh asks) are
   accumulated into, on leaf boxes only; with ifpghtarg >= 1 the leaf
   interpolants of pot (and grad, hess) are evaluated at targs(2,ntarg) into
   pote(nd,ntarg), grade(nd,2,ntarg), hesse(nd,3,ntarg), overwritten
   (boxfgt.f:207-276, 1494-1563).  The colleague arrays itree(iptr(6)),
   itree(iptr(7)) are recomputed as the reference does (boxfgt.f:516-528);
   timeinfo(1:20) is zeroed and filled with per-stage seconds. */
void boxfgt_(const int *nd, const int *ndim, const double *delta, const double *eps, const int *ipoly,
             int *iperiod, const int *norder, const int *npbox, int *nboxes, int *nlevels, int *ltree,
             int *itree, int *iptr, double *centers, double *boxsize, const double *fvals, const int *ifpgh,
             double *pot, double *grad, double *hess, const int *ifnewtree, const int *ntarg,
             const double *targs, const int *ifpghtarg, double *pote, double *grade, double *hesse,
             double *timeinfo);

/* No counterpart in the reference.  Precision mode of boxfgt_ (which has no
   precision argument): BFGT_PREC_FP64 (the default) or BFGT_PREC_SPLIT.  The
   environment variable BFGT_PRECISION=split selects split before the first
   call.  A call that split precision cannot serve (norder other than 8 and 16,
   npw > 64, eps < 1e-11) runs in FP64. */
int bfgt_set_default_precision(int precision);

/* No counterpart in the reference.  boxfgt_ and bfgt_boxfgt keep the plans
   (step-0 precomputation and device tables) of their last few argument sets,
   16 by default or BFGT_PLAN_CACHE (0 turns the cache off).  A plan is found
   again when nd, delta, eps, ipoly, iperiod, norder, precision, nboxes,
   nlevels, ltree, the device, iptr, itree up to its colleague arrays, centers
   and boxsize all equal, bit for bit, those it was built from (the cache keeps
   a copy of them); on a hit the colleague arrays are written back as a fresh
   plan would leave them and timeinfo(1) is the lookup time.  Calls into the cache
   are serialised by a mutex.  bfgt_plan_cache_clear frees the cached plans;
   bfgt_plan_cache_info gives out[0] entries, out[1] capacity, out[2] hits,
   out[3] misses (out must hold 4). */
int bfgt_plan_cache_clear(void);
int bfgt_plan_cache_info(int64_t *out);

/* No counterpart in the reference.  Bytes the last boxfgt_ / bfgt_boxfgt call
   copied host to device (out[0]) and device to host (out[1]).  pot, grad and
   hess runs that are all +0.0 on the host (the reference's callers zero pot
   before each call, hpots/hpots2dadap.f:97-101, 321-325) are cleared on the
   device instead of uploaded, with the same result bit for bit. */
int bfgt_boxfgt_last_bytes(double *out);

/* Last error message of this thread ("" when the last call succeeded). */
const char *bfgt_last_error(void);

/* Same as boxfgt_ with values instead of references and a precision mode.
   Replaces bfgt/boxfgt.f:5-286 for callers that are not Fortran. Returns a
   BFGT_* status. */
int bfgt_boxfgt(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes, int nlevels,
                int ltree, int *itree, const int *iptr, const double *centers, const double *boxsize,
                const double *fvals, double *pot, double *timeinfo, int precision);

/* ---- plan API (device-resident boxfgt) ---------------------------------- */
typedef struct bfgt_plan_s *bfgt_plan;

/* Builds the step-0 precomputation of bfgt/boxfgt.f:472-703 (cutoff level,
   plane-wave nodes, 1D tables, interaction lists) for one tree, delta, eps,
   norder, ipoly and nd, and uploads it to the current CUDA device.  itree's
   colleague arrays are recomputed in place as boxfgt does. */
int bfgt_plan_create(bfgt_plan *plan, int nd, double delta, double eps, int ipoly, int iperiod, int norder,
                     int nboxes, int nlevels, int ltree, int *itree, const int *iptr, const double *centers,
                     const double *boxsize, int precision);

/* Steps 1-6 of bfgt/boxfgt.f:720-1071 on device arrays laid out as
   fvals(nd,norder**2,nboxes) and pot(nd,norder**2,nboxes); pot is accumulated
   into on leaf boxes.  stream is a cudaStream_t (NULL = default stream).
   Asynchronous: returns after the launches are queued. */
int bfgt_plan_execute(bfgt_plan plan, const double *d_fvals, double *d_pot, void *stream);
/* (Every entry point that takes device arrays returns BFGT_ERR_ARG, before
   launching anything, for an array that is not device memory of the plan's
   device.) */

/* Same transform on host arrays: uploads the leaf values, runs, and adds the
   result into the host pot (the reference-facing form of a planned call). */
int bfgt_plan_execute_host(bfgt_plan plan, const double *fvals, double *pot, void *stream);

/* Replaces the ifpgh = 2, 3 branches of bfgt/boxfgt.f steps 5 and 6
   (gnd_pw2pgh -> g2d_pw2pg / g2d_pw2pgh, bfgt_pwrouts.f:309-375, 608-784;
   gnd_tens_prod_to_pghloc -> g2d_tens_prod_to_pgloc / _pghloc,
   bfgt_local.f:379-552) on device arrays: pot += K fvals, and for ifpgh >= 2
   grad(nd,2,norder**2,nboxes) += its gradient (x, y), for ifpgh = 3 also
   hess(nd,3,norder**2,nboxes) += its hessian (xx, xy, yy), on leaf boxes.
   ifpgh = 1 is bfgt_plan_execute (grad and hess may then be NULL).  The first
   call with ifpgh >= 2 uploads the derivative tables (synchronous); later
   calls only queue kernels on stream. */
int bfgt_plan_execute_pgh(bfgt_plan plan, int ifpgh, const double *d_fvals, double *d_pot, double *d_grad,
                          double *d_hess, void *stream);

/* The same on host arrays (leaf boxes copied in and out). */
int bfgt_plan_execute_pgh_host(bfgt_plan plan, int ifpgh, const double *fvals, double *pot, double *grad,
                               double *hess, void *stream);

/* Replaces bfgt/boxfgt.f step 11 (1494-1563: treedata_trans_nd and
   treedata_evalt_nd, common/tree_data_routs_nd.f:16-60, 710-780, with the
   target sort of pts_tree_sort, common/pts_tree_nd.f:1226-1260) on device
   arrays: out(nd*ncomp, ntarg) = the leaf interpolants of
   vals(nd*ncomp, norder**2, nboxes) at targs(2, ntarg), overwritten.  ncomp is
   1 for pot, 2 for grad, 3 for hess.  A target belongs to the leaf reached
   from the root by child 1 + (x >= cx) + 2 (y >= cy).  Grows its device
   scratch (coefficients and target leaves) on the first call that needs more. */
int bfgt_plan_eval_targets(bfgt_plan plan, int ncomp, const double *d_vals, int ntarg, const double *d_targs,
                           double *d_out, void *stream);

/* No counterpart in the reference (boxfgt has no adjoint; this is the
   differentiation entry point).  Applies the transpose of this plan's discrete
   transform on device arrays: fbar(nd,norder**2,nboxes) += K^T potbar on leaf
   boxes, where pot += K fvals is what bfgt_plan_execute computes, so that
   sum(potbar * K f) = sum(f * K^T potbar) over leaf values.  For
   J = 0.5*|K f - g|^2 the gradient dJ/dfvals is K^T (K f - g).  Same precision
   mode as the plan.  The first call builds the transposed tables (host
   precomputation and device allocation, synchronous); later calls only queue
   kernels on stream. */
int bfgt_plan_execute_adjoint(bfgt_plan plan, const double *d_potbar, double *d_fbar, void *stream);

/* The same on host arrays (leaf boxes copied in and out, as in
   bfgt_plan_execute_host). */
int bfgt_plan_execute_adjoint_host(bfgt_plan plan, const double *potbar, double *fbar, void *stream);

/* No counterpart in the reference (the Fortran boxfgt allocates its own
   workspace on every call).  Runs the same transform as bfgt_plan_execute
   without allocating anything: the plane-wave scratch (partial expansions of
   the leaf chunks and the cutoff-box expansions) comes from one static device
   array of bfgt_noalloc_scratch_bytes() (32 MiB) per GPU, held until exit.
   For callers that may not allocate device memory while they step: a solver
   whose own memory manager owns the device (a caching allocator, pools
   reserved at start-up), or a stepping loop that cannot afford the device
   stalls of cudaMalloc/cudaFree.  Plans whose scratch need
   (bfgt_plan_noalloc_need) exceeds the array are rejected with
   BFGT_ERR_CAPACITY.  The first call on a device looks up the array's address
   (cudaGetSymbolAddress) and should come before any stream capture; the
   address is kept for the life of the process, so a process that calls
   cudaDeviceReset must not use this entry point afterwards.  Calls that
   overlap on the GPU share, and race on, the array. */
int bfgt_plan_execute_noalloc(bfgt_plan plan, const double *d_fvals, double *d_pot, void *stream);
int bfgt_noalloc_scratch_bytes(size_t *bytes);
int bfgt_plan_noalloc_need(bfgt_plan plan, size_t *bytes);

/* Capture bfgt_plan_execute for these device buffers into a CUDA graph and
   replay it with bfgt_plan_graph_launch. */
int bfgt_plan_graph_capture(bfgt_plan plan, const double *d_fvals, double *d_pot, void *stream);
int bfgt_plan_graph_launch(bfgt_plan plan, void *stream);

/* Device milliseconds per stage, summed over every bfgt_plan_execute on this
   plan since the previous call (CUDA events recorded on the execute stream):
   out[0] leaf values -> cutoff expansions (steps 1+2), out[1] fixed-order
   reduction, out[2] cutoff translation (step 3), out[3] cutoff expansions ->
   leaf values (steps 4+5), out[4] near field (step 6), out[5] total, out[6]
   number of executes summed.  Waits for the last of them.  out must hold 8. */
int bfgt_plan_stage_ms(bfgt_plan plan, double *out);

/* Creates n sets of stage events ahead of a timed loop (one set per execute). */
int bfgt_plan_reserve_events(bfgt_plan plan, int n);

/* Plan scalars: out[0]=npwlevel (boxfgt.f:137-150), out[1]=npw, out[2]=nlevstart,
   out[3]=nlevend, out[4]=regime (0 periodic Fourier, 1 PW + near field,
   2 near field only), out[5]=nleafbox, out[6]=number of PW leaves,
   out[7]=number of near-field target leaves, out[8]=number of near-field
   interactions, out[9]=mnlist1, out[10]=internal iperiod, out[11]=number of
   plane-wave chunks (CTAs of the form and eval kernels), out[12]=kernel
   launches per execute, out[13]/out[14]=FP64 form/eval tile shape in use
   (100 tm + 10 tn + tiles per lane; 0 for split plans), out[15]=split
   kernel shapes in use (1000 when the eval kernel runs the chunks' column
   halves + 100 eval step group + 10 x-contraction tiles per form thread + 1
   when the form kernel stages Y as float2; 0 for FP64 plans).  out must hold
   16 ints. */
int bfgt_plan_info(bfgt_plan plan, int *out);

/* Algorithmic work of one execute (every real operation counted once, split
   slices not multiplied): out[0]=FLOP, out[1]=compulsory HBM bytes (leaf fvals
   read + pot read/write), out[2]=tensor-core FLOP issued (split mode; every
   slice product counted), out[3]=leaf points x nd, out[4..7]=FLOP of the form,
   eval, near-field and translation stages, out[8..10]=compulsory bytes of the
   form, eval and near-field stages, out[11..12]=tensor-core FLOP issued by the
   form and eval stages, out[13..14]=bytes bfgt_plan_execute_host moves host to
   device and device to host (leaf boxes only), out[15]=bytes the last
   host-array execute actually uploaded: accumulator runs (pot, grad, hess)
   that are all +0.0 on the host are cleared on the device instead of copied,
   as when the caller zeroes pot before each call.  out must hold 16. */
int bfgt_plan_work(bfgt_plan plan, double *out);

/* No counterpart in the reference.  Autotuner of the kernels' compiled
   shapes: times every shape of the form and eval kernels that fits this plan
   on its own work (on scratch arrays it allocates; synchronous) and keeps the
   fastest.  FP64 plans: the tile shapes, remembered for plans of the same
   (norder, npw, nd) created later in the process.  Split-precision plans: Y
   staged as float2 or double2 and 1 or 2 x-contraction tiles per thread in
   the form kernel, step groups of 8, 4 or 2 and whole chunks or their column
   halves in the eval kernel (for this plan only).  FP64 shapes give the same sums to rounding, split shapes the same
   bits.  report (may be NULL) receives
   the best form and eval ms per launch and the numbers of shapes timed.  A
   batch or a captured graph keeps the shapes its plans had when it was made:
   tune first. */
int bfgt_plan_autotune(bfgt_plan plan, void *stream, double *report);

/* Waits for the device and reports failures of earlier executes on this plan:
   BFGT_ERR_TIMEOUT if a bounded device-side wait of the tensor-core pipeline
   gave up (the results of that execute are not valid), BFGT_ERR_CUDA on a
   device error.  Clears the flag. */
int bfgt_plan_check(bfgt_plan plan);

/* No counterpart in the reference.  Sets the poll limit of the bounded
   device-side waits of this plan's tensor-core kernels (default 2^26 polls,
   restored by passing 0xFFFFFFFF).  A wait that reaches the limit makes the
   kernel stop issuing tensor-core work, drain what is in flight, free its
   tensor memory and return; bfgt_plan_check then reports BFGT_ERR_TIMEOUT and
   that execute's result is invalid.  A limit of 0 makes every such wait give
   up at once (used to test the error path).  No effect on FP64 plans. */
int bfgt_plan_set_wait_limit(bfgt_plan plan, unsigned int polls);

int bfgt_plan_destroy(bfgt_plan plan);

/* ---- batches of plans --------------------------------------------------- */
/* No counterpart in the reference: its solvers call boxfgt once per density,
   species and time node with its own delta (hpots/hpots2dadap.f:329-346,
   4018-4102).  A batch runs the transforms of several plans (independent
   trees, deltas, eps, orders, nd) together: the split-precision form and eval
   stages of all plans go through one launch per kernel variant driven by a
   device-side list of (plan, chunk) work items, and the cutoff translations
   and the near field of all plans through one launch each; FP64 plans run
   their form and eval stages as launches of their own.  The plans must stay
   alive (and on the current device) while the batch exists.  The leaf arrays
   are packed: plan i's fvals(nd_i,norder_i**2,nboxes_i) and pot start at
   element offsets[i] of the batch arrays (bfgt_batch_layout). */
typedef struct bfgt_batch_s *bfgt_batch;
int bfgt_batch_create(bfgt_batch *batch, int nplans, const bfgt_plan *plans);
/* offsets: nplans + 1 element offsets (the last is the packed length). */
int bfgt_batch_layout(bfgt_batch batch, int64_t *offsets);
/* pot += K_i fvals for every plan i, on the packed device arrays; asynchronous. */
int bfgt_batch_execute(bfgt_batch batch, const double *d_fvals, double *d_pot, void *stream);
/* The transposed transforms of every plan (bfgt_plan_execute_adjoint),
   batched the same way, on packed arrays with the same layout:
   fbar += K_i^T potbar for every plan i.  The first call builds the plans'
   transposed tables and the batch over them (synchronous). */
int bfgt_batch_execute_adjoint(bfgt_batch batch, const double *d_potbar, double *d_fbar, void *stream);
/* Capture bfgt_batch_execute for these buffers into a CUDA graph / replay it. */
int bfgt_batch_graph_capture(bfgt_batch batch, const double *d_fvals, double *d_pot, void *stream);
int bfgt_batch_graph_launch(bfgt_batch batch, void *stream);
/* Stage milliseconds summed over the executes since the last call, as
   bfgt_plan_stage_ms. */
int bfgt_batch_stage_ms(bfgt_batch batch, double *out);
/* out[0]=plans, out[1]=kernel launches per execute, out[2]/out[3]=form/eval
   work items (chunks), out[4]=translation blocks, out[5]=near-field blocks.
   out must hold 8. */
int bfgt_batch_info(bfgt_batch batch, int *out);
/* bfgt_plan_check on every plan of the batch. */
int bfgt_batch_check(bfgt_batch batch);
int bfgt_batch_destroy(bfgt_batch batch);

/* ---- host-side plan introspection (no device needed) ------------------- */
/* Builds only the host half of a plan (tables and lists) and copies out the
   interaction lists and near-field band patterns so that they can be compared
   bit for bit with another implementation of bfgt/boxfgt.f step 0.  Any output
   pointer may be NULL.  list1 is written as list1(mnlist1_cap, nboxes), listpw
   as listpw(8, nboxes), ind_loc as ind_loc(2, norder+1, -6:6, 0:nlevels) and
   tab_loc as tab_loc(norder, norder, -6:6, 0:nlevels). info as bfgt_plan_info. */
int bfgt_host_plan_dump(int nd, double delta, double eps, int ipoly, int iperiod, int norder, int nboxes,
                        int nlevels, int ltree, int *itree, const int *iptr, const double *centers,
                        const double *boxsize, int *info, int *ifpwexp, int *nlist1, int *list1,
                        int mnlist1_cap, int *nlistpw, int *listpw, int *ind_loc, double *tab_loc, double *ts,
                        double *ws);

/* ---- caller-side tree generator ---------------------------------------- */
/* Adaptive level-restricted quad tree on [-L/2,L/2]^2 resolving
   f(x) = sum_g a_g exp(-|x-c_g|^2 / w_g^2) (gauss: ng rows of {cx,cy,w,a}),
   with the tail criterion of common/tree_vol_coeffs_nd.f:689-780 (iptype=2,
   given eta) and 2:1 balance, as vol_tree_build (tree_vol_coeffs_nd.f:440)
   produces; maxlev caps the depth (0 = no cap), minlev forces uniform
   refinement down to that level.  Returns a handle; sizes via
   bfgt_tree_sizes, arrays via bfgt_tree_export (itree(ltree), iptr(8),
   centers(2,nboxes), boxsize(0:nlevels), fvals(nd=1,norder**2,nboxes)). */
typedef struct bfgt_tree_s *bfgt_tree;
int bfgt_tree_build_gauss(bfgt_tree *tree, int ipoly, int iperiod, double eps, double boxlen, int norder,
                          double eta, int ng, const double *gauss, int minlev, int maxlev);
/* Uniform tree of depth nlev (4**nlev leaves), f evaluated as above. */
int bfgt_tree_build_uniform(bfgt_tree *tree, int ipoly, int iperiod, double boxlen, int norder, int nlev,
                            int ng, const double *gauss);
int bfgt_tree_sizes(bfgt_tree tree, int *nboxes, int *nlevels, int *ltree);
int bfgt_tree_export(bfgt_tree tree, int *itree, int *iptr, double *centers, double *boxsize, double *fvals);
int bfgt_tree_free(bfgt_tree tree);

#ifdef __cplusplus
}
#endif
#endif
