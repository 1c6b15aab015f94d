// lce_capi.cu -- the extern "C" boundary (include/lceqcd_gpu.h).
//
// A context owns one CUDA stream, one device allocation holding the fields of
// all its chains, a chain table, the device-resident run state (RNG pass
// counter, validation-stream position, status bits, per-chain gauge-fixing
// state) and FP64 partial-sum buffers.  Update routines are queued as one
// kernel per parity pass followed by one finalize kernel; lce_sweep captures
// its whole pass sequence once per measflag into a CUDA graph and replays it.
// The RNG counters live on the device, so a replayed graph draws fresh
// numbers every time.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <array>
#include <deque>
#include <map>
#include <tuple>
#include <string>
#include <vector>

#include "lce_internal.hpp"

using namespace lce;

namespace {

thread_local std::string g_create_error;

struct Pass {
  unsigned char kind;
  int eo, mu;
  bool end;  // last pass of its routine
};

}  // namespace

void lce::set_thread_error(const std::string& msg) { g_create_error = msg; }

// one autotune candidate: a sweep form and, for the per-pass forms, the tile
// shape (threads per block, sites per thread), with its timed samples
struct TuneForm {
  int form, bs, spt, occ;  // occ: resident threads per SM of the register cap (0: the default)
  std::vector<float> ms;
};

struct lce_ctx {
  int device = 0;
  int prec = LCE_PREC_F32;
  int rng = LCE_RNG_PHILOX;
  int nchains = 0;
  int n_link_or = 0, n_higgs_metro = 0;
  int eo_flip = 0;        // a z-slab's local parity of whole-lattice parity 0
  int s_lo = 0, site_off = 0;  // a z-slab's first visited site and Philox site offset (PassArgs)
  int stream_nh = 0;      // a z-slab's whole-lattice sites per parity (validation stream slots)
  int agauge_hits = 1;  // 1: f/agauge.f, 3: f/agauge1.f in lce_sweep
  std::vector<lce_params> params;
  std::vector<ChainDev> ch;
  // prefix over chains of the tiles of one pass, for tiles of 128, 256, 512
  // and 448 sites (kTileSites; tile = threads per block x sites per thread);
  // tiles of kBlock sites (blk) serve the persistent form
  std::vector<int> tiles[kTileTables];
  std::vector<int>& blk = tiles[1];
  int max_nh = 0, max_L3 = 0;
  ChainDev* ch_d = nullptr;
  int* tiles_d[kTileTables] = {nullptr, nullptr, nullptr, nullptr};
  int* blk_d = nullptr;   // = tiles_d[1]
  // finalize reduction: per tile table, the prefix over chains of chunks of
  // kChunkTiles tiles, and the chunk sums [chunk][kMaxSlots][kNQ]
  std::vector<int> chunks[kTileTables];
  int* chunks_begin_d[kTileTables] = {nullptr, nullptr, nullptr, nullptr};
  double* chunks_d = nullptr;
  CtxState* st_d = nullptr;
  ChainState* cst_d = nullptr;
  lce_meas* meas_d = nullptr;
  double* part_d = nullptr;
  int part_slots = 0;
  size_t slot_stride = 0;
  double* totals_d = nullptr;
  double* scratch_d = nullptr;
  size_t scratch_n = 0;
  void* fields_d = nullptr;
  double* stream_d = nullptr;
  size_t stream_n = 0;
  void* staging_d = nullptr;
  size_t staging_bytes = 0;
  // asynchronous uploads (lce_upload_stage / lce_upload_apply): copy stream,
  // two staging slots (links then A of the largest chain, each), the events
  // that order the two streams around each slot, and the staged uploads not
  // yet applied (oldest first: slot, chain, field selector)
  cudaStream_t copy = nullptr;
  cudaEvent_t staged_ev[2] = {nullptr, nullptr}, free_ev[2] = {nullptr, nullptr};
  void* async_d = nullptr;
  size_t async_slot = 0;  // bytes per slot
  int next_slot = 0;
  std::deque<std::array<int, 3>> staged;
  void* flush_d = nullptr;
  size_t flush_bytes = 0;
  void* gsave_d = nullptr;  // G_prev during a warm-started gauge fixing
  void* fa_d = nullptr;     // Fourier-accelerated fixing: FFT fields and the step transform
  size_t fa_bytes = 0;
  std::map<std::pair<int, int>, cudaGraphExec_t> fa_exec;
  cudaStream_t own = nullptr, stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // per-pass timing inside a sweep graph (lce_profile_sweep): a side stream
  // with its fork/join events and one timing event per pass boundary
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  std::vector<cudaEvent_t> prof_ev;
  // instantiated sweep graphs by (form, threads per block, sites per thread,
  // register-cap occupancy, measflag)
  std::map<std::tuple<int, int, int, int, int, int>, cudaGraphExec_t> sweep_graphs;
  GridBar* bar_d = nullptr;
  int persist_grid = 0;
  int sweep_mode = LCE_SWEEP_AUTO;   // requested
  int mode = LCE_SWEEP_AUTO;         // in use (AUTO while tuning)
  int tile_req = 0;                  // requested threads per block (0: tuned under AUTO, else 256)
  int tile_bs = kBlock, tile_spt = 1;  // tile shape of the per-pass kernels in use
  int tile_occ = 0;                    // its register-cap occupancy (0: the default)
  std::vector<TuneForm> tune;        // autotune candidates and their samples
  std::map<std::pair<int, int>, cudaGraphExec_t> gf_exec;
  std::string err;
};

namespace {

int fail(lce_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  else g_create_error = msg;
  return code;
}

int cuda_fail(lce_ctx* c, cudaError_t e, const char* where) {
  return fail(c, LCE_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

size_t link_bytes(int prec) { return prec == LCE_PREC_F64 ? 32 : 16; }
size_t real_bytes(int prec) { return prec == LCE_PREC_F64 ? 8 : 4; }
size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// f/paraminit.f:44-47 and :150-153, in the precision of the fields
template <typename T>
void couplings_t(double beta, double x, double y, double out[3]) {
  const T pi = (T)2.0 * (T)std::acos((T)0.0);
  const T sigma = (T)3.1759114;
  const T b = (T)beta, xx = (T)x, yy = (T)y;
  const T beta_a = b;
  const T beta_2 = beta_a * ((T)3 + (T)8 * yy / (b * b) - sigma * ((T)4 + (T)5 * xx) / ((T)2 * pi * b) -
                             (((T)20 * xx - (T)10 * (xx * xx)) * ((T)std::log((T)1.5 * b) + (T)0.09) + (T)8.7 +
                              (T)11.6 * xx) /
                                 (((T)2 * (pi * pi)) * (b * b)));
  out[0] = beta_a;
  out[1] = beta_2;
  out[2] = xx * b;
}

bool valid_params(const lce_params& p, std::string& why) {
  for (int i = 0; i < 3; ++i)
    if (p.L[i] < 2 || (p.L[i] & 1)) {
      why = "lattice extents must be even and >= 2";
      return false;
    }
  double v = (double)p.L[0] * p.L[1] * p.L[2];
  if (v / 2 > 1.0e9) {
    why = "lattice too large for 32-bit site indices";
    return false;
  }
  if (p.precision != LCE_PREC_F32 && p.precision != LCE_PREC_F64) {
    why = "precision must be LCE_PREC_F32 or LCE_PREC_F64";
    return false;
  }
  if (p.rng != LCE_RNG_PHILOX && p.rng != LCE_RNG_STREAM) {
    why = "rng must be LCE_RNG_PHILOX or LCE_RNG_STREAM";
    return false;
  }
  if (!(p.beta > 0)) {
    why = "beta must be positive";
    return false;
  }
  if (p.imode != 0 && p.imode != 1) {
    why = "imode must be 0 or 1";
    return false;
  }
  if (p.sweep_mode < LCE_SWEEP_AUTO || p.sweep_mode > LCE_SWEEP_DIRECT) {
    why = "sweep_mode must be LCE_SWEEP_AUTO, LCE_SWEEP_PASSES, LCE_SWEEP_PASSES2, LCE_SWEEP_PERSISTENT or "
          "LCE_SWEEP_DIRECT";
    return false;
  }
  if (p.tile_threads != 0 && p.tile_threads != 128 && p.tile_threads != 256 && p.tile_threads != 448 &&
      p.tile_threads != 512) {
    why = "tile_threads must be 0 (tuned), 128, 256, 448 or 512";
    return false;
  }
  if (p.tile_registers != 0 && !(p.tile_registers == 56 && p.tile_threads == 128 && p.precision == LCE_PREC_F32)) {
    why = "tile_registers must be 0, or 56 with tile_threads = 128 in FP32";
    return false;
  }
  if (p.gf_angle != LCE_GF_ACOS && p.gf_angle != LCE_GF_ATAN2) {
    why = "gf_angle must be LCE_GF_ACOS or LCE_GF_ATAN2";
    return false;
  }
  if (!(p.lambda > 0) || !(p.alpha >= 0)) {
    why = "lambda must be positive and alpha non-negative";
    return false;
  }
  if (p.agauge_hits != 0 && p.agauge_hits != 1 && p.agauge_hits != 3) {
    why = "agauge_hits must be 1 (f/agauge.f) or 3 (f/agauge1.f)";
    return false;
  }
  if (p.n_link_or < 0 || p.n_higgs_metro < 0 || 4 + 6 + 2 * p.n_higgs_metro + 6 * p.n_link_or > kMaxSlots) {
    why = "too many extra update passes per sweep";
    return false;
  }
  return true;
}

int status_check(lce_ctx* c) {
  CtxState st;
  CK(cudaMemcpyAsync(&st, c->st_d, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st.status) {
    unsigned int z = 0;
    CK(cudaMemcpy(&c->st_d->status, &z, sizeof(z), cudaMemcpyHostToDevice));
    if (st.status & kStatusStreamExhausted) return fail(c, LCE_ERR_STREAM, "validation uniform stream exhausted");
    if (st.status & kStatusBarrierTimeout) {
      // leave the barrier in a clean state for the next launch
      CK(cudaMemset(c->bar_d, 0, sizeof(GridBar)));
      return fail(c, LCE_ERR_CUDA, "persistent sweep: a grid barrier timed out");
    }
    return fail(c, LCE_ERR_NAN, "non-finite value in a measurement reduction");
  }
  return LCE_OK;
}

int nslots_of(unsigned char kind) {
  switch (kind) {
    case kHiggsHB: return 7;
    case kHiggsOR: return 1;
    case kHiggsMetro: return 4;
    case kLinkHB: return 7;
    case kLinkHB3: return 21;
    default: return 1;
  }
}

// Philox passes a pass kind consumes (one per hit)
int philox_passes(unsigned char kind) { return kind == kLinkHB3 ? 3 : 1; }

void expand(unsigned char kind, std::vector<Pass>& out) {
  if (kind <= kHiggsMetro) {
    out.push_back({kind, 0, 0, false});
    out.push_back({kind, 1, 0, true});
  } else {
    for (int eo = 0; eo < 2; ++eo)
      for (int mu = 0; mu < 3; ++mu) out.push_back({kind, eo, mu, eo == 1 && mu == 2});
  }
}

}  // namespace

// The finalize combine's routine groups.  A scan over the slots in order adds
// each slot's totals to the accumulator of its class (Higgs: ahiggs1-3;
// links: agauge, agauge1, link overrelaxation) and, at a slot flagged as the
// end of a routine, normalises the accumulator and clears it.  Group g is
// the set of slots such a scan adds before the g-th end (in slot order), so
// that groups can be summed and normalised independently.  Flags: the last
// Higgs group (a2, a4, akin are written by every Higgs group, the last
// one's stay), the last group of each kind ({agauge, agauge1} share plaq and
// acc_gauge), the ahiggs1 groups.
void lce::fin_groups(FinalizeArgs& f) {
  std::memset(f.gid, kNoGroup, sizeof(f.gid));
  std::memset(f.gflags, 0, sizeof(f.gflags));
  std::memset(f.gbeg, 0, sizeof(f.gbeg));
  std::memset(f.gend, 0, sizeof(f.gend));
  f.ngroups = 0;
  f.nmetro = 0;
  std::vector<int> members[2];
  int last_higgs = -1, last_kind[6] = {-1, -1, -1, -1, -1, -1};
  for (int i = 0; i < f.nslots; ++i) {
    const int kind = f.kinds[i] & 0x7f, cls = kind <= kHiggsMetro ? 0 : 1;
    members[cls].push_back(i);
    if (!(f.kinds[i] & kKindEnd)) continue;
    const int g = f.ngroups++;
    for (int j : members[cls]) f.gid[j] = (unsigned char)g;
    f.gbeg[g] = (unsigned char)members[cls].front();
    f.gend[g] = (unsigned char)i;
    members[cls].clear();
    if (kind == kHiggsMetro) f.gflags[g] |= kGrpMetro, ++f.nmetro;
    if (kind <= kHiggsMetro) last_higgs = g;
    last_kind[kind == kLinkHB3 ? kLinkHB : kind] = g;
  }
  if (last_higgs >= 0) f.gflags[last_higgs] |= kGrpHiggsLast;
  for (int k = 0; k < 6; ++k)
    if (last_kind[k] >= 0) f.gflags[last_kind[k]] |= kGrpKindLast;
}

namespace {

// Queue the passes of the given routines and one finalize kernel.
// events: optional array receiving an event record after every pass.
// The passes of a list of routines, queued one at a time: enq_begin plans
// them, enq_pass launches pass i, enq_end queues the finalize reduction.
struct Enq {
  std::vector<Pass> passes;
  FinalizeArgs f;
  const std::vector<int>* blk = nullptr;
  int* blk_d = nullptr;
  int spt = 1, bs = kBlock, occ = 0;
  int measflag = 0;
  bool fuse = false;
  unsigned long long soff = 0;
  unsigned int poff = 0;
  int slot = 0;
  int prev_slot = -1;  // reduction slot of the previous pass, or -1
  bool rb = false;     // reduce-behind (the one-site-per-thread kernels)
  // graphs of several sweeps (sweep_graph): the previous sweep's finalize,
  // run by an extra block of this queue's first pass; defer_out: leave this
  // queue's finalize in f for the next queue instead of launching it
  const FinalizeArgs* defer_in = nullptr;
  bool defer_out = false;
};

// reduce-behind blocks of a pass: enough warps for one level-1 item each, at
// most kReduceBlocks blocks
constexpr int kReduceBlocks = 64;

// index of the chain table for tiles of bs * spt sites (128, 256 or 512)
int tile_index(int bs, int spt) {
  const int t = bs * spt;
  return t == 128 ? 0 : (t == 256 ? 1 : (t == 512 ? 2 : 3));
}

// poff0, soff0: the queue's RNG offsets from the counters' values (nonzero
// for the later sweeps of a graph of several sweeps)
void enq_begin(lce_ctx* c, const std::vector<unsigned char>& routines, int measflag, bool fuse_renorm, int bs,
               int spt, int occ, Enq& q, unsigned int poff0 = 0, unsigned long long soff0 = 0) {
  const int ti = tile_index(bs, spt);
  q.blk = &c->tiles[ti];
  q.blk_d = c->tiles_d[ti];
  q.spt = spt;
  q.bs = bs;
  q.occ = occ;
  q.measflag = measflag;
  q.fuse = fuse_renorm;
  q.passes.clear();
  for (unsigned char r : routines) expand(r, q.passes);
  FinalizeArgs& f = q.f;
  std::memset(&f, 0, sizeof(f));
  f.chains = c->ch_d;
  f.blk_begin = q.blk_d;
  f.st = c->st_d;
  f.cst = c->cst_d;
  f.meas = c->meas_d;
  f.part = c->part_d;
  f.slot_stride = c->slot_stride;
  f.totals = c->totals_d;
  f.nchains = c->nchains;
  f.single = c->prec == LCE_PREC_F32;
  f.chunk_begin = c->chunks_begin_d[ti];
  f.chunks = c->chunks_d;
  f.nchunks = c->chunks[ti].back();
  f.ntiles0 = c->tiles[ti][1];
  q.soff = soff0;
  q.poff = poff0;
  q.slot = 0;
  q.prev_slot = -1;
  q.rb = spt == 1;
}

int enq_pass(lce_ctx* c, Enq& q, size_t i) {
  const Pass& ps = q.passes[i];
  const int nblocks = q.blk->back();
  const bool reduce = q.measflag == 1 || ps.kind == kHiggsMetro;
  if (reduce && q.slot >= c->part_slots) return fail(c, LCE_ERR_INVALID, "too many reduction slots");
  PassArgs a{};
  a.chains = c->ch_d;
  a.blk_begin = q.blk_d;
  a.spt = q.spt;
  a.bs = q.bs;
  a.occ = q.occ;
  a.st = c->st_d;
  a.cst = c->cst_d;
  a.part = reduce ? c->part_d + (size_t)q.slot * c->slot_stride : nullptr;
  a.stream = c->rng == LCE_RNG_STREAM ? c->stream_d : nullptr;
  a.stream_n = c->stream_n;
  a.stream_off = q.soff;
  a.pass_off = q.poff;
  a.nchains = c->nchains;
  a.eo = ps.eo ^ c->eo_flip;
  a.fuse_renorm = q.fuse ? 1 : 0;
  a.s_lo = c->s_lo;
  a.site_off = c->site_off;
  a.stream_nh = c->stream_nh;
  // the first pass of a queue follows whatever the stream ran before (an
  // earlier queue's finalize may still be advancing the RNG counters); the
  // later passes follow pass kernels of this queue only
  a.rng_early = i > 0 ? 1 : 0;
  a.trigger_late = i == 0 ? 1 : 0;
  // level 1 of the previous pass's slot in extra blocks of this launch
  a.ntiles = nblocks;
  int grid = nblocks;
  if (q.rb && q.prev_slot >= 0) {
    a.rb_slot = q.prev_slot | (tile_index(q.bs, q.spt) << 8);
    a.rb_nitems = q.f.nchunks;
    const int wpb = q.bs / 32;
    grid += std::min(kReduceBlocks, (a.rb_nitems + wpb - 1) / wpb);
  }
  if (i == 0 && q.defer_in) {
    // the previous sweep's finalize in one extra block (sweep_graph checked
    // that this pass is ahiggs2 with one site per thread and no reduce-behind)
    if (c->prec == LCE_PREC_F64) launch_higgs_fin<double>(a, *q.defer_in, grid + 1, c->stream);
    else launch_higgs_fin<float>(a, *q.defer_in, grid + 1, c->stream);
  } else if (ps.kind <= kHiggsMetro) {
    if (c->prec == LCE_PREC_F64) launch_higgs<double>(ps.kind, a, grid, c->stream);
    else launch_higgs<float>(ps.kind, a, grid, c->stream);
  } else {
    const int mode = ps.kind == kLinkHB ? 0 : (ps.kind == kLinkOR ? 1 : 2);
    if (c->prec == LCE_PREC_F64) launch_link<double>(mode, ps.mu, a, grid, c->stream);
    else launch_link<float>(mode, ps.mu, a, grid, c->stream);
  }
  q.prev_slot = reduce ? q.slot : -1;
  if (reduce) {
    q.f.kinds[q.slot] = (unsigned char)(ps.kind | (ps.end ? kKindEnd : 0));
    ++q.slot;
  }
  if (c->nchains == 1) q.soff += (unsigned long long)nslots_of(ps.kind) * (c->stream_nh ? c->stream_nh : c->ch[0].nh);
  q.poff += philox_passes(ps.kind);
  return LCE_OK;
}

int enq_end(lce_ctx* c, Enq& q) {
  q.f.nslots = q.slot;
  q.f.npasses = q.poff;
  q.f.nstream = c->rng == LCE_RNG_STREAM ? q.soff : 0;
  // reduce-behind: every slot but the last pass's was summed by the pass after it
  q.f.pre = !q.rb ? 0 : (q.prev_slot >= 0 ? q.slot - 1 : q.slot);
  fin_groups(q.f);
  if (q.defer_out) {
    // run by the next queue's first pass; inside a graph of sweeps the
    // counters advance at its last finalize only
    q.f.npasses = 0;
    q.f.nstream = 0;
    return LCE_OK;
  }
  launch_finalize(q.f, c->stream);
  CK(cudaGetLastError());
  return LCE_OK;
}

// bs, spt, occ: the tile shape (bs = 0: the context's shape in use)
int enqueue(lce_ctx* c, const std::vector<unsigned char>& routines, int measflag, bool fuse_renorm,
            cudaEvent_t* events = nullptr, int bs = 0, int spt = 0, int occ = 0) {
  Enq q;
  if (!bs) {
    bs = c->tile_bs;
    spt = c->tile_spt;
    occ = c->tile_occ;
  }
  enq_begin(c, routines, measflag, fuse_renorm, bs, spt, occ, q);
  for (size_t i = 0; i < q.passes.size(); ++i) {
    if (int rc = enq_pass(c, q, i)) return rc;
    if (events) CK(cudaEventRecord(events[i], c->stream));
  }
  return enq_end(c, q);
}

std::vector<unsigned char> sweep_routines(const lce_ctx* c);

// Queue the passes of the given routines as one cooperative persistent kernel
// (plan of passes, reduction slots and stream offsets as in enqueue).
template <typename R>
int enqueue_persistent(lce_ctx* c, const std::vector<unsigned char>& routines, int measflag, bool fuse_renorm) {
  std::vector<Pass> passes;
  for (unsigned char r : routines) expand(r, passes);
  if ((int)passes.size() > kMaxSlots) return fail(c, LCE_ERR_INVALID, "too many passes for one persistent sweep");
  PersistArgs a;
  std::memset(&a, 0, sizeof(a));
  PassArgs& b = a.base;
  b.chains = c->ch_d;
  b.blk_begin = c->blk_d;
  b.st = c->st_d;
  b.cst = c->cst_d;
  b.stream = c->rng == LCE_RNG_STREAM ? c->stream_d : nullptr;
  b.stream_n = c->stream_n;
  b.nchains = c->nchains;
  b.fuse_renorm = fuse_renorm ? 1 : 0;
  b.spt = 1;
  b.bs = kBlock;
  b.occ = 0;
  b.s_lo = c->s_lo;
  b.site_off = c->site_off;
  b.stream_nh = c->stream_nh;
  b.rng_early = 0;
  b.trigger_late = 0;
  FinalizeArgs& f = a.fin;
  f.chains = c->ch_d;
  f.blk_begin = c->blk_d;
  f.st = c->st_d;
  f.cst = c->cst_d;
  f.meas = c->meas_d;
  f.part = c->part_d;
  f.slot_stride = c->slot_stride;
  f.totals = c->totals_d;
  f.nchains = c->nchains;
  f.single = c->prec == LCE_PREC_F32;
  f.chunk_begin = c->chunks_begin_d[1];
  f.chunks = c->chunks_d;
  f.nchunks = c->chunks[1].back();
  f.ntiles0 = c->tiles[1][1];
  unsigned long long soff = 0;
  unsigned int poff = 0;
  int slot = 0;
  for (size_t i = 0; i < passes.size(); ++i) {
    const Pass& ps = passes[i];
    const bool reduce = measflag == 1 || ps.kind == kHiggsMetro;
    if (reduce && slot >= c->part_slots) return fail(c, LCE_ERR_INVALID, "too many reduction slots");
    a.pass_off[i] = (unsigned short)poff;
    poff += philox_passes(ps.kind);
    a.plan[i] = PlanEntry{ps.kind, (unsigned char)(ps.eo ^ c->eo_flip), (unsigned char)ps.mu,
                          reduce ? (unsigned char)slot : kNoSlot};
    a.stream_off[i] = soff;
    if (reduce) {
      f.kinds[slot] = (unsigned char)(ps.kind | (ps.end ? kKindEnd : 0));
      ++slot;
    }
    if (c->nchains == 1) soff += (unsigned long long)nslots_of(ps.kind) * c->ch[0].nh;
  }
  f.nslots = slot;
  f.npasses = poff;
  f.nstream = c->rng == LCE_RNG_STREAM ? soff : 0;
  f.pre = 0;
  fin_groups(f);
  a.bar = c->bar_d;
  a.ntiles = c->blk.back();
  a.npasses = (int)passes.size();
  const int grid = std::max(1, std::min(c->persist_grid, a.ntiles));
  CK(launch_persistent<R>(a, grid, c->stream));
  return LCE_OK;
}

constexpr size_t kTuneSamples = 3;

// Graphs of several sweeps defer each sweep's finalize (but the last) into an
// extra block of the next sweep's first pass (higgs_fin_kernel): a single
// chain of at most 8 chunks (the single-chain finalize), the per-pass form
// with one site per thread and a tile shape that kernel is compiled for.
bool sweeps_defer_finalize(const lce_ctx* c, int form, int bs, int spt, int occ) {
  if (form != LCE_SWEEP_PASSES || spt != 1 || occ != 0 || c->nchains != 1) return false;
  if (c->chunks[tile_index(bs, spt)].back() > 8) return false;
  return c->prec == LCE_PREC_F64 ? bs == 256 : (bs == 128 || bs == 256 || bs == 448 || bs == 512);
}

// nrep sweeps with deferred finalizes: sweep r's passes take the RNG offsets
// r x (one sweep's advance) from the counters, which only the last sweep's
// finalize advances (by nrep sweeps' worth)
int enqueue_sweeps_deferred(lce_ctx* c, int nrep, int mf, int bs) {
  const std::vector<unsigned char> r = sweep_routines(c);
  std::vector<Pass> passes;
  for (unsigned char k : r) expand(k, passes);
  unsigned int per = 0;
  unsigned long long nst = 0;
  for (const Pass& ps : passes) {
    per += philox_passes(ps.kind);
    nst += (unsigned long long)nslots_of(ps.kind) * (c->stream_nh ? c->stream_nh : c->ch[0].nh);
  }
  FinalizeArgs prev;
  for (int k = 0; k < nrep; ++k) {
    Enq q;
    q.defer_in = k > 0 ? &prev : nullptr;
    q.defer_out = k < nrep - 1;
    enq_begin(c, r, mf, true, bs, 1, 0, q, per * (unsigned)k, nst * (unsigned long long)k);
    for (size_t i = 0; i < q.passes.size(); ++i)
      if (int rc = enq_pass(c, q, i)) return rc;
    if (int rc = enq_end(c, q)) return rc;
    if (q.defer_out) prev = q.f;
  }
  return LCE_OK;
}

// Runs of sweeps (lce_sweeps) replay a graph of kSweepsPerGraph sweeps: inside
// one graph a sweep's first pass launches programmatically behind the
// previous sweep's finalize (and waits for it before reading the RNG
// counters), instead of after a graph boundary.
constexpr int kSweepsPerGraph = 8;

// The instantiated graph of nrep sweeps in the given form (built once per
// form, measflag and nrep).  The persistent form falls back to the per-pass
// form under LCE_SWEEP_AUTO if it cannot be captured on this device.
int sweep_graph(lce_ctx* c, int form, int bs, int spt, int occ, int mf, cudaGraphExec_t* out, int nrep = 1) {
  if (form == LCE_SWEEP_PERSISTENT) bs = kBlock, spt = 1, occ = 0;
  cudaGraphExec_t* slot = &c->sweep_graphs[std::make_tuple(form, bs, spt, occ, mf, nrep)];
  if (!*slot) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = LCE_OK;
    if (nrep > 1 && sweeps_defer_finalize(c, form, bs, spt, occ)) rc = enqueue_sweeps_deferred(c, nrep, mf, bs);
    else
      for (int r = 0; r < nrep && rc == LCE_OK; ++r) {
        if (form == LCE_SWEEP_PERSISTENT)
          rc = c->prec == LCE_PREC_F64 ? enqueue_persistent<double>(c, sweep_routines(c), mf, true)
                                       : enqueue_persistent<float>(c, sweep_routines(c), mf, true);
        else
          rc = enqueue(c, sweep_routines(c), mf, true, nullptr, bs, spt, occ);
      }
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    cudaError_t ei = cudaSuccess;
    if (ec == cudaSuccess) {
      if (rc == LCE_OK) ei = cudaGraphInstantiate(slot, g, 0);
      cudaGraphDestroy(g);
    }
    if (rc) return rc;
    const cudaError_t e = ec != cudaSuccess ? ec : ei;
    if (e != cudaSuccess) {
      *slot = nullptr;
      cudaGetLastError();
      if (form == LCE_SWEEP_PERSISTENT && c->sweep_mode == LCE_SWEEP_AUTO) {
        c->err = std::string("persistent sweep unavailable: ") + cudaGetErrorString(e);
        c->mode = LCE_SWEEP_PASSES;
        c->tune.clear();
        return sweep_graph(c, LCE_SWEEP_PASSES, c->tile_bs, c->tile_spt, c->tile_occ, mf, out, nrep);
      }
      return cuda_fail(c, e, "sweep graph capture");
    }
  }
  *out = *slot;
  return LCE_OK;
}

std::vector<unsigned char> sweep_routines(const lce_ctx* c) {
  std::vector<unsigned char> r = {kHiggsHB, kHiggsOR};
  for (int i = 0; i < c->n_higgs_metro; ++i) r.push_back(kHiggsMetro);
  r.push_back(c->agauge_hits == 3 ? kLinkHB3 : kLinkHB);
  for (int i = 0; i < c->n_link_or; ++i) r.push_back(kLinkOR);
  return r;
}

int routine_call(lce_ctx* c, unsigned char kind, int measflag, float* accept, bool renorm) {
  int rc = enqueue(c, {kind}, measflag, renorm);
  if (rc) return rc;
  if (!accept) return LCE_OK;
  rc = status_check(c);
  if (rc) return rc;
  lce_meas m;
  CK(cudaMemcpy(&m, c->meas_d, sizeof(m), cudaMemcpyDeviceToHost));
  switch (kind) {
    case kHiggsHB: *accept = (float)m.acc_hb; break;
    case kHiggsOR: *accept = (float)m.acc_or; break;
    case kHiggsMetro: *accept = (float)m.acc_metro; break;
    case kLinkHB: *accept = (float)m.acc_gauge; break;
    case kLinkHB3: *accept = (float)m.acc_gauge; break;
    default: *accept = (float)m.acc_link_or; break;
  }
  return LCE_OK;
}

int ensure_staging(lce_ctx* c, size_t bytes) {
  if (c->staging_bytes >= bytes) return LCE_OK;
  if (c->staging_d) CK(cudaFree(c->staging_d));
  c->staging_d = nullptr;
  c->staging_bytes = 0;
  CK(cudaMalloc(&c->staging_d, bytes));
  c->staging_bytes = bytes;
  return LCE_OK;
}

void* field_ptr(const ChainDev& ch, int which, bool links) {
  if (which == LCE_FIELDS) return links ? ch.u : ch.a;
  return links ? ch.uf : ch.af;
}

template <typename Rin>
int upload_t(lce_ctx* c, int chain, int which, const Rin* u, const Rin* a, long ld) {
  if (chain < 0 || chain >= c->nchains || (which != LCE_FIELDS && which != LCE_FIELDS_FIXED))
    return fail(c, LCE_ERR_INVALID, "upload: bad chain or field selector");
  const ChainDev& ch = c->ch[chain];
  if (ld < ch.nh) return fail(c, LCE_ERR_INVALID, "upload: ld smaller than L1*L2*L3/2");
  const int nh = ch.nh;
  if (u) {
    void* dst = field_ptr(ch, which, true);
    const bool direct = (sizeof(Rin) == real_bytes(c->prec));
    if (direct) {
      CK(cudaMemcpy2DAsync(dst, (size_t)nh * 4 * sizeof(Rin), u, (size_t)ld * 4 * sizeof(Rin),
                           (size_t)nh * 4 * sizeof(Rin), 6, cudaMemcpyHostToDevice, c->stream));
    } else {
      int rc = ensure_staging(c, (size_t)6 * c->max_nh * 4 * sizeof(double));
      if (rc) return rc;
      CK(cudaMemcpy2DAsync(c->staging_d, (size_t)nh * 4 * sizeof(Rin), u, (size_t)ld * 4 * sizeof(Rin),
                           (size_t)nh * 4 * sizeof(Rin), 6, cudaMemcpyHostToDevice, c->stream));
      if (c->prec == LCE_PREC_F64) launch_links_in<Rin, double>((const Rin*)c->staging_d, dst, nh, c->stream);
      else launch_links_in<Rin, float>((const Rin*)c->staging_d, dst, nh, c->stream);
    }
  }
  if (a) {
    void* dst = field_ptr(ch, which, false);
    int rc = ensure_staging(c, (size_t)6 * c->max_nh * 4 * sizeof(double));
    if (rc) return rc;
    CK(cudaMemcpy2DAsync(c->staging_d, (size_t)nh * 3 * sizeof(Rin), a, (size_t)ld * 3 * sizeof(Rin),
                         (size_t)nh * 3 * sizeof(Rin), 2, cudaMemcpyHostToDevice, c->stream));
    if (c->prec == LCE_PREC_F64) launch_higgs_in<Rin, double>((const Rin*)c->staging_d, dst, nh, c->stream);
    else launch_higgs_in<Rin, float>((const Rin*)c->staging_d, dst, nh, c->stream);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return LCE_OK;
}

template <typename Rout>
int download_t(lce_ctx* c, int chain, int which, Rout* u, Rout* a, long ld) {
  if (chain < 0 || chain >= c->nchains || (which != LCE_FIELDS && which != LCE_FIELDS_FIXED))
    return fail(c, LCE_ERR_INVALID, "download: bad chain or field selector");
  const ChainDev& ch = c->ch[chain];
  if (ld < ch.nh) return fail(c, LCE_ERR_INVALID, "download: ld smaller than L1*L2*L3/2");
  const int nh = ch.nh;
  if (u) {
    const void* src = field_ptr(ch, which, true);
    if (sizeof(Rout) == real_bytes(c->prec)) {
      CK(cudaMemcpy2DAsync(u, (size_t)ld * 4 * sizeof(Rout), src, (size_t)nh * 4 * sizeof(Rout),
                           (size_t)nh * 4 * sizeof(Rout), 6, cudaMemcpyDeviceToHost, c->stream));
    } else {
      int rc = ensure_staging(c, (size_t)6 * c->max_nh * 4 * sizeof(double));
      if (rc) return rc;
      if (c->prec == LCE_PREC_F64) launch_links_out<double, Rout>(src, (Rout*)c->staging_d, nh, c->stream);
      else launch_links_out<float, Rout>(src, (Rout*)c->staging_d, nh, c->stream);
      CK(cudaMemcpy2DAsync(u, (size_t)ld * 4 * sizeof(Rout), c->staging_d, (size_t)nh * 4 * sizeof(Rout),
                           (size_t)nh * 4 * sizeof(Rout), 6, cudaMemcpyDeviceToHost, c->stream));
    }
  }
  if (a) {
    const void* src = field_ptr(ch, which, false);
    int rc = ensure_staging(c, (size_t)6 * c->max_nh * 4 * sizeof(double));
    if (rc) return rc;
    if (c->prec == LCE_PREC_F64) launch_higgs_out<double, Rout>(src, (Rout*)c->staging_d, nh, c->stream);
    else launch_higgs_out<float, Rout>(src, (Rout*)c->staging_d, nh, c->stream);
    CK(cudaMemcpy2DAsync(a, (size_t)ld * 3 * sizeof(Rout), c->staging_d, (size_t)nh * 3 * sizeof(Rout),
                         (size_t)nh * 3 * sizeof(Rout), 2, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return LCE_OK;
}

// one z-slab of a decomposed lattice: its chain's first and last planes are
// halos, the update passes visit the planes between them
struct SlabInfo {
  int site_off;  // site index of the first local site in the whole lattice (plane z0 - 1)
  int eo_flip;   // local parity = whole-lattice parity ^ eo_flip
  int nh;        // sites per parity of the whole lattice
};

lce_ctx* create_impl(const lce_params* p, int n, const SlabInfo* slab = nullptr) {
  g_create_error.clear();
  if (!p || n < 1) {
    fail(nullptr, LCE_ERR_INVALID, "create: null params or no chains");
    return nullptr;
  }
  for (int i = 0; i < n; ++i) {
    std::string why;
    if (!valid_params(p[i], why)) {
      fail(nullptr, LCE_ERR_INVALID, "create: chain " + std::to_string(i) + ": " + why);
      return nullptr;
    }
    if (p[i].precision != p[0].precision || p[i].rng != p[0].rng || p[i].device != p[0].device ||
        p[i].n_link_or != p[0].n_link_or || p[i].n_higgs_metro != p[0].n_higgs_metro ||
        p[i].agauge_hits != p[0].agauge_hits) {
      fail(nullptr, LCE_ERR_INVALID, "create: chains of a batch must share precision, rng, device and composition");
      return nullptr;
    }
  }
  if (n > 1 && p[0].rng == LCE_RNG_STREAM) {
    fail(nullptr, LCE_ERR_UNSUPPORTED, "create: validation streams need a single-chain context");
    return nullptr;
  }
  lce_ctx* c = new lce_ctx();
  c->device = p[0].device;
  c->prec = p[0].precision;
  c->rng = p[0].rng;
  c->nchains = n;
  c->n_link_or = p[0].n_link_or;
  c->n_higgs_metro = p[0].n_higgs_metro;
  c->agauge_hits = p[0].agauge_hits == 3 ? 3 : 1;
  c->eo_flip = slab ? slab->eo_flip : 0;
  c->s_lo = slab ? p[0].L[0] * p[0].L[1] / 2 : 0;
  c->site_off = slab ? slab->site_off : 0;
  c->stream_nh = slab ? slab->nh : 0;
  c->params.assign(p, p + n);
  auto bail = [&](cudaError_t e, const char* where) -> lce_ctx* {
    g_create_error = std::string(where) + ": " + cudaGetErrorString(e);
    lce_destroy(c);
    return nullptr;
  };
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return bail(e, "cudaSetDevice");
  e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(e, "cudaStreamCreate");
  c->stream = c->own;
  if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess) return bail(e, "cudaEventCreate");
  if ((e = cudaEventCreate(&c->ev1)) != cudaSuccess) return bail(e, "cudaEventCreate");

  // chain table and field layout
  const size_t lb = link_bytes(c->prec), rb = real_bytes(c->prec);
  size_t off = 0;
  std::vector<size_t> offs;
  for (auto& t : c->tiles) t.assign(1, 0);
  for (int i = 0; i < n; ++i) {
    ChainDev d;
    std::memset(&d, 0, sizeof(d));
    d.L1 = p[i].L[0];
    d.L2 = p[i].L[1];
    d.L3 = p[i].L[2];
    d.hx = d.L1 / 2;
    d.nxy = d.L1 * d.L2 / 2;
    d.nh = d.nxy * d.L3;
    d.dhx = make_fastdiv((uint32_t)d.hx);
    d.dnxy = make_fastdiv((uint32_t)d.nxy);
    double cp[3];
    lce_couplings(&p[i], cp);
    if (c->prec == LCE_PREC_F32) {
      d.beta = (float)p[i].beta;
      d.lambda = (float)p[i].lambda;
      d.alpha = (float)p[i].alpha;
      d.limit_or = (float)p[i].limit_or;
    } else {
      d.beta = p[i].beta;
      d.lambda = p[i].lambda;
      d.alpha = p[i].alpha;
      d.limit_or = p[i].limit_or;
    }
    d.beta_a = cp[0];
    d.beta_2 = cp[1];
    d.beta_4 = cp[2];
    if (c->prec == LCE_PREC_F32) {
      d.inv_beta2 = 1.0f / (float)cp[1];
      d.cxval0 = 1.0f / (float)cp[1] / 2.0f;
    } else {
      d.inv_beta2 = 1.0 / cp[1];
      d.cxval0 = 1.0 / cp[1] / 2.0;
    }
    d.imode = p[i].imode;
    d.gf_angle = p[i].gf_angle;
    d.key0 = (uint32_t)p[i].seed;
    d.key1 = (uint32_t)(p[i].seed >> 32);

    offs.push_back(off);
    off += 2 * (align256((size_t)6 * d.nh * lb) + align256((size_t)6 * d.nh * rb)) + align256((size_t)2 * d.nh * lb);
    c->ch.push_back(d);
    const int nvis = slab ? d.nh - 2 * d.nxy : d.nh;  // sites a pass visits per parity
    for (int t = 0; t < kTileTables; ++t) c->tiles[t].push_back(c->tiles[t].back() + ceil_div(nvis, kTileSites[t]));
    c->max_nh = std::max(c->max_nh, d.nh);
    c->max_L3 = std::max(c->max_L3, d.L3);
  }
  if ((e = cudaMalloc(&c->fields_d, off)) != cudaSuccess) return bail(e, "cudaMalloc(fields)");
  for (int i = 0; i < n; ++i) {
    char* b = (char*)c->fields_d + offs[i];
    ChainDev& d = c->ch[i];
    const size_t ul = align256((size_t)6 * d.nh * lb), al = align256((size_t)6 * d.nh * rb);
    d.u = b;
    d.a = b + ul;
    d.uf = b + ul + al;
    d.af = b + 2 * ul + al;
    d.g = b + 2 * ul + 2 * al;
  }
  if ((e = cudaMemset(c->fields_d, 0, off)) != cudaSuccess) return bail(e, "cudaMemset(fields)");
  if ((e = cudaMalloc(&c->ch_d, sizeof(ChainDev) * n)) != cudaSuccess) return bail(e, "cudaMalloc(chains)");
  if ((e = cudaMemcpy(c->ch_d, c->ch.data(), sizeof(ChainDev) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return bail(e, "cudaMemcpy(chains)");
  for (int t = 0; t < kTileTables; ++t) {
    if ((e = cudaMalloc(&c->tiles_d[t], sizeof(int) * (n + 1))) != cudaSuccess) return bail(e, "cudaMalloc(tiles)");
    if ((e = cudaMemcpy(c->tiles_d[t], c->tiles[t].data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
      return bail(e, "cudaMemcpy(tiles)");
    c->chunks[t].assign(1, 0);
    for (int i = 0; i < n; ++i)
      c->chunks[t].push_back(c->chunks[t].back() + ceil_div(c->tiles[t][i + 1] - c->tiles[t][i], kChunkTiles));
    if ((e = cudaMalloc(&c->chunks_begin_d[t], sizeof(int) * (n + 1))) != cudaSuccess)
      return bail(e, "cudaMalloc(chunk table)");
    if ((e = cudaMemcpy(c->chunks_begin_d[t], c->chunks[t].data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
      return bail(e, "cudaMemcpy(chunk table)");
  }
  {
    // 128-site tiles (table 0) make the most chunks
    const size_t nd = (size_t)c->chunks[0].back() * kMaxSlots * kNQ;
    if ((e = cudaMalloc(&c->chunks_d, sizeof(double) * nd)) != cudaSuccess) return bail(e, "cudaMalloc(chunk sums)");
  }
  c->blk_d = c->tiles_d[1];
  if ((e = cudaMalloc(&c->st_d, sizeof(CtxState))) != cudaSuccess) return bail(e, "cudaMalloc(state)");
  if ((e = cudaMemset(c->st_d, 0, sizeof(CtxState))) != cudaSuccess) return bail(e, "cudaMemset(state)");
  if ((e = cudaMalloc(&c->cst_d, sizeof(ChainState) * n)) != cudaSuccess) return bail(e, "cudaMalloc(cstate)");
  {
    std::vector<ChainState> cs(n);
    for (int i = 0; i < n; ++i) {
      std::memset(&cs[i], 0, sizeof(ChainState));
      cs[i].delta = p[i].delta0;
    }
    if ((e = cudaMemcpy(c->cst_d, cs.data(), sizeof(ChainState) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
      return bail(e, "cudaMemcpy(cstate)");
  }
  if ((e = cudaMalloc(&c->meas_d, sizeof(lce_meas) * n)) != cudaSuccess) return bail(e, "cudaMalloc(meas)");
  if ((e = cudaMalloc(&c->bar_d, sizeof(GridBar))) != cudaSuccess) return bail(e, "cudaMalloc(barrier)");
  if ((e = cudaMemset(c->bar_d, 0, sizeof(GridBar))) != cudaSuccess) return bail(e, "cudaMemset(barrier)");
  c->sweep_mode = p[0].sweep_mode;
  c->mode = p[0].sweep_mode;
  c->persist_grid = c->prec == LCE_PREC_F64 ? persistent_grid<double>() : persistent_grid<float>();
  if (c->persist_grid <= 0 && c->sweep_mode == LCE_SWEEP_PERSISTENT) {
    g_create_error = "create: the persistent sweep kernel cannot be made resident on this device";
    lce_destroy(c);
    return nullptr;
  }
  // tile shape: FP32 contexts tune threads per block (128, 256, 512) and sites
  // per thread under AUTO unless tile_threads fixes the block; the FP64
  // validation path and z-slabs use kBlock threads
  c->tile_req = (c->prec == LCE_PREC_F32 && !slab) ? p[0].tile_threads : kBlock;
  c->tile_bs = c->tile_req ? c->tile_req : kBlock;
  c->tile_spt = c->mode == LCE_SWEEP_PASSES2 ? 2 : 1;
  if (c->tile_spt == 2 && c->tile_bs > 256) c->tile_bs = kBlock;  // (448, 2), (512, 2) are not compiled
  const bool reg56 = !slab && p[0].tile_registers == 56;
  if (reg56) {
    c->tile_bs = 128;
    c->tile_spt = 1;
    c->tile_occ = 1152;
  }
  if (c->mode == LCE_SWEEP_AUTO) {
    const int bss[4] = {128, 256, 448, 512};
    for (int b : bss) {
      if (reg56) {
        c->tune.push_back(TuneForm{LCE_SWEEP_PASSES, 128, 1, 1152, {}});
        break;
      }
      if (c->tile_req && b != c->tile_req) continue;
      if (c->prec == LCE_PREC_F64 && b != kBlock) continue;
      c->tune.push_back(TuneForm{LCE_SWEEP_PASSES, b, 1, 0, {}});
      if (b <= 256) c->tune.push_back(TuneForm{LCE_SWEEP_PASSES2, b, 2, 0, {}});
    }
    // Not candidates, measured slower on the B200 at 64^3 and 128^3 (still
    // selectable): the 56-register 128-thread form (tile_registers = 56,
    // 71.1 / 381.1 us per sweep against 64.7 / 374-377 us) and the direct
    // launches without a graph (LCE_SWEEP_DIRECT, 66.0 / 380.0 us against
    // 64.6 / 377.5 us with the same tile).
    if (c->persist_grid > 0) c->tune.push_back(TuneForm{LCE_SWEEP_PERSISTENT, kBlock, 1, 0, {}});
  }
  if ((e = cudaMemset(c->meas_d, 0, sizeof(lce_meas) * n)) != cudaSuccess) return bail(e, "cudaMemset(meas)");
  c->part_slots = std::max(6, 4 + 6 + 2 * c->n_higgs_metro + 6 * c->n_link_or);
  c->slot_stride = (size_t)c->tiles[0].back() * kNQ;  // the most tiles: 128 sites each
  if ((e = cudaMalloc(&c->part_d, sizeof(double) * c->slot_stride * c->part_slots)) != cudaSuccess)
    return bail(e, "cudaMalloc(partials)");
  if ((e = cudaMalloc(&c->totals_d, sizeof(double) * (size_t)n * kMaxSlots * kNQ)) != cudaSuccess)
    return bail(e, "cudaMalloc(totals)");
  {
    // the reduce-behind blocks' buffers
    static_assert(sizeof(CtxState::rb_chunk_begin) / sizeof(int*) == kTileTables, "one chunk table per tile table");
    CtxState st{};
    st.rb_part = c->part_d;
    st.rb_slot_stride = c->slot_stride;
    for (int t = 0; t < kTileTables; ++t) st.rb_chunk_begin[t] = c->chunks_begin_d[t];
    st.rb_chunks = c->chunks_d;
    st.rb_totals = c->totals_d;
    if ((e = cudaMemcpy(c->st_d, &st, sizeof(st), cudaMemcpyHostToDevice)) != cudaSuccess)
      return bail(e, "cudaMemcpy(state)");
  }
  c->scratch_n = (size_t)2 * ceil_div(2L * c->max_nh, 256) + (size_t)32 * c->max_L3 + 64;
  if ((e = cudaMalloc(&c->scratch_d, sizeof(double) * c->scratch_n)) != cudaSuccess)
    return bail(e, "cudaMalloc(scratch)");
  if (c->max_L3 * 14 * sizeof(double) > 48 * 1024) {
    // correlator kernel stages the slice sums in shared memory
    if (c->max_L3 * 14 * sizeof(double) > 200 * 1024) {
      g_create_error = "create: L3 too large for the correlator kernel";
      lce_destroy(c);
      return nullptr;
    }
  }
  return c;
}

int get_slices(lce_ctx* c, int chain, double*& out) {
  const ChainDev& ch = c->ch[chain];
  double* slices = c->scratch_d;
  out = c->scratch_d + (size_t)14 * ch.L3;
  if (c->prec == LCE_PREC_F64) launch_slice_sums<double>(c->ch_d + chain, ch.L3, slices, c->stream);
  else launch_slice_sums<float>(c->ch_d + chain, ch.L3, slices, c->stream);
  launch_correlators(slices, ch.L1, ch.L2, ch.L3, out, c->stream);
  CK(cudaGetLastError());
  return LCE_OK;
}

// it_flags >= 0: the iterative form (LCE_ITGF_* flags, step), else overrelaxation
int gf_loop(lce_ctx* c, int chain, double* theta, int* iters, int max_iters, int track = 0, int it_flags = -1,
            double step = 0.0) {
  const ChainDev& ch = c->ch[chain];
  // bounded on the device in every case; no cap requested means 10^6
  const int cap = max_iters > 0 ? max_iters : 1000000;
  ChainState cs;
  CK(cudaMemcpyAsync(&cs, c->cst_d + chain, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  cs.gf_done = 0;
  cs.gf_iters = 0;
  cs.gf_cap = cap;
  cs.gf_theta = 1.0e4;
  if (it_flags >= 0) cs.gf_step = step;
  CK(cudaMemcpyAsync(c->cst_d + chain, &cs, sizeof(cs), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double* part = c->scratch_d;
  int batch = 8;
  while (true) {
    // graph key: form (0 overrelaxation, 1 + flags iterative), batch, tracking
    auto key = std::make_pair(chain, ((it_flags + 1) << 10) + 2 * batch + (track ? 1 : 0));
    auto it = c->gf_exec.find(key);
    if (it == c->gf_exec.end()) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < batch; ++k) {
        if (it_flags >= 0) {
          if (c->prec == LCE_PREC_F64)
            launch_it_iteration<double>(c->ch_d + chain, c->cst_d + chain, it_flags, 1, part, ch.nh, c->stream);
          else
            launch_it_iteration<float>(c->ch_d + chain, c->cst_d + chain, it_flags, 1, part, ch.nh, c->stream);
        } else if (c->prec == LCE_PREC_F64) {
          launch_gf_iteration<double>(c->ch_d + chain, c->cst_d + chain, track, part, ch.nh, c->stream);
        } else {
          launch_gf_iteration<float>(c->ch_d + chain, c->cst_d + chain, track, part, ch.nh, c->stream);
        }
      }
      CK(cudaStreamEndCapture(c->stream, &g));
      cudaGraphExec_t ex;
      cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate(gauge fixing)");
      it = c->gf_exec.emplace(key, ex).first;
    }
    const int before = cs.gf_iters;
    CK(cudaGraphLaunch(it->second, c->stream));
    CK(cudaMemcpyAsync(&cs, c->cst_d + chain, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (cs.gf_done) break;
    if (cs.gf_iters <= before) return fail(c, LCE_ERR_CUDA, "gauge fixing: a batch of iterations made no progress");
    if (batch < 256) batch *= 2;
  }
  if (theta) *theta = cs.gf_theta;
  if (iters) *iters = cs.gf_iters;
  if (!std::isfinite(cs.gf_theta)) return fail(c, LCE_ERR_NAN, "gauge fixing: theta is not finite");
  if (cs.gf_theta > ch.limit_or) return fail(c, LCE_ERR_GF_NOT_CONVERGED, "gauge fixing: iteration cap reached");
  return LCE_OK;
}

// one allocation for the largest chain, allocated once: the captured graphs
// of every chain keep pointing into it
size_t fa_vcap(const lce_ctx* c) { return 2 * (size_t)c->max_nh; }

int fa_buffers(lce_ctx* c) {
  if (c->fa_d) return LCE_OK;
  const size_t need = fa_buffer_bytes(fa_vcap(c));
  if (cudaMalloc(&c->fa_d, need) != cudaSuccess) {
    c->fa_d = nullptr;
    return fail(c, LCE_ERR_NOMEM, "Fourier-accelerated fixing buffers");
  }
  c->fa_bytes = need;
  fa_init_table(c->fa_d, fa_vcap(c), c->stream);
  CK(cudaGetLastError());
  return LCE_OK;
}

// Fourier-accelerated iterations on U_f (tracking G) until theta <= limit or
// the cap; same graph batching and progress guard as gf_loop; cg: the
// conjugate-gradient form (its direction starts afresh)
int fa_loop(lce_ctx* c, int chain, double step, double limit, double* theta, int* iters, int cap, bool cg = false) {
  const ChainDev& ch = c->ch[chain];
  int rc = fa_buffers(c);
  if (rc) return rc;
  ChainState cs;
  CK(cudaMemcpyAsync(&cs, c->cst_d + chain, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  cs.gf_done = 0;
  cs.gf_iters = 0;
  cs.gf_cap = cap;
  cs.gf_theta = 1.0e4;
  cs.gf_limit = limit;
  cs.gf_step = step;
  CK(cudaMemcpyAsync(c->cst_d + chain, &cs, sizeof(cs), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double* part = c->scratch_d;
  if (cg) fa_cg_reset(c->fa_d, fa_vcap(c), c->stream);
  int batch = 4;
  while (true) {
    auto key = std::make_pair(chain, 2 * batch + (cg ? 1 : 0));
    auto it = c->fa_exec.find(key);
    if (it == c->fa_exec.end()) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < batch; ++k) {
        if (c->prec == LCE_PREC_F64)
          launch_fa_iteration<double>(c->ch_d + chain, ch, c->cst_d + chain, step, c->fa_d, fa_vcap(c), part,
                                      nullptr, 1, true, true, cg, c->stream);
        else
          launch_fa_iteration<float>(c->ch_d + chain, ch, c->cst_d + chain, step, c->fa_d, fa_vcap(c), part,
                                     nullptr, 1, true, true, cg, c->stream);
      }
      const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
      const std::string fe = fa_take_error();
      if (!fe.empty()) {
        if (ec == cudaSuccess) cudaGraphDestroy(g);
        cudaGetLastError();
        return fail(c, LCE_ERR_CUDA, "Fourier-accelerated fixing: " + fe);
      }
      if (ec != cudaSuccess) return cuda_fail(c, ec, "cudaStreamEndCapture(Fourier-accelerated fixing)");
      cudaGraphExec_t ex;
      cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate(Fourier-accelerated fixing)");
      it = c->fa_exec.emplace(key, ex).first;
    }
    const int before = cs.gf_iters;
    CK(cudaGraphLaunch(it->second, c->stream));
    CK(cudaMemcpyAsync(&cs, c->cst_d + chain, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (cs.gf_done) break;
    if (cs.gf_iters <= before)
      return fail(c, LCE_ERR_CUDA, "Fourier-accelerated fixing: a batch of iterations made no progress");
    if (batch < 64) batch *= 2;
  }
  if (theta) *theta = cs.gf_theta;
  if (iters) *iters = cs.gf_iters;
  if (!std::isfinite(cs.gf_theta)) return fail(c, LCE_ERR_NAN, "Fourier-accelerated fixing: theta is not finite");
  return LCE_OK;
}

}  // namespace

// ====================================================================== C ABI
// ------------------------------------------------------------------ z-slabs
// A lattice split along z into slabs (the reference's domain decomposition,
// f/topology.f with dimproc = (1, 1, n), and its halo exchange around every
// pass of f/staples.f / f/a_force.f), each slab a one-chain context on its
// own device or sharing one.  Slab k holds the whole lattice's planes
// z0 - 1 .. z0 + nz (z0 = k nz): its first and last local planes are halos,
// the update passes visit the nz planes between them, and the Philox
// counters use whole-lattice site indices, so a decomposed run draws the
// uniforms of the undecomposed one and reproduces its fields bit for bit.
// After every pass the written field's parity is exchanged: slab k copies
// the last interior plane of slab k-1 into its plane 0 and the first
// interior plane of slab k+1 into its plane nz+1 (periodic), on its own
// stream, ordered by events (peer copies between devices).  Gauge fixing and
// the correlators gather per-slab sums on slab 0's device (g_d).
struct lce_slabs {
  std::vector<lce_ctx*> slab;
  std::vector<cudaEvent_t> ev_pass, ev_copy, ev_sum;
  cudaEvent_t ev_chk = nullptr;
  double* g_d = nullptr;  // slab 0's device: theta sums [n], slice sums [14 L3], correlators [7 L3 + 5]
  void* fft_d = nullptr;  // slab 0's device: the whole lattice's two transformed fields (Fourier fixing)
  void* cg_d = nullptr;   // slab 0's device: the conjugate-gradient form's whole-lattice buffers (FaSlabCg)
  FaSlabCg cgw{};
  int L[3] = {0, 0, 0};
  int nz = 0, nxy = 0, prec = LCE_PREC_F32;
  double delta = 0.0;  // ahiggs1 step of the whole lattice (every slab holds a copy)
};

namespace {

int slabs_fail(int code, const std::string& m) {
  set_thread_error(m);
  return code;
}
#define SCK(call)                                                                                   \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) return slabs_fail(LCE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// a slab context's error, made the thread's last error (lce_last_error(NULL))
int slab_rc(lce_ctx* c, int rc) {
  if (rc && !c->err.empty()) set_thread_error(c->err);
  return rc;
}

// device address of local plane z of a slab's field at local parity p: the
// links U_mu (f = mu) or component k of the Higgs field (f = -1); fixed:
// the gauge-fixed copies U_f, A_f
// f: a link direction 0-2, 3 for the gauge transform G, 4 for the Fourier
// iteration's step transform g (FP64), -1 for the Higgs field
// 5 for component k of the conjugate-gradient direction (FP32)
size_t slab_elem_bytes(const lce_ctx* c, int f) {
  return f == 5 ? 4 : (f == 4 ? 32 : (f >= 0 ? link_bytes(c->prec) : real_bytes(c->prec)));
}
int slab_components(int f) { return f == 5 || f < 0 ? 3 : 1; }
char* slab_plane(lce_ctx* c, int f, int p, int z, int k, bool fixed = false) {
  const ChainDev& d = c->ch[0];
  if (f == 5) return (char*)fa_sdir_ptr(c->fa_d, fa_vcap(c)) + (((size_t)(k * 2 + p)) * d.nh + (size_t)z * d.nxy) * 4;
  if (f == 4) return (char*)fa_gstep_ptr(c->fa_d, fa_vcap(c)) + ((size_t)p * d.nh + (size_t)z * d.nxy) * 32;
  if (f == 3) return (char*)d.g + ((size_t)p * d.nh + (size_t)z * d.nxy) * link_bytes(c->prec);
  if (f >= 0)
    return (char*)(fixed ? d.uf : d.u) + (((size_t)(f * 2 + p)) * d.nh + (size_t)z * d.nxy) * link_bytes(c->prec);
  return (char*)(fixed ? d.af : d.a) + (((size_t)(p * 3 + k)) * d.nh + (size_t)z * d.nxy) * real_bytes(c->prec);
}

// one plane of an exchange: slab k's local plane zd of field f (a link
// direction, or -1 for the Higgs field) at whole-lattice parity pg, from
// plane zs of its neighbour k + dk (dk = -1 or +1, periodic)
struct PlaneCopy {
  int dk, zs, zd, f, pg;
  bool fixed;
};

int slab_copy_plane(lce_ctx* c, lce_ctx* cj, const PlaneCopy& q, size_t nxy) {
  const int ps = q.pg ^ cj->eo_flip, pd = q.pg ^ c->eo_flip;
  const size_t bytes = nxy * slab_elem_bytes(c, q.f);
  for (int comp = 0; comp < slab_components(q.f); ++comp) {
    void* dst = slab_plane(c, q.f, pd, q.zd, comp, q.fixed);
    const void* src = slab_plane(cj, q.f, ps, q.zs, comp, q.fixed);
    if (c->device == cj->device) SCK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
    else SCK(cudaMemcpyPeerAsync(dst, c->device, src, cj->device, bytes, c->stream));
  }
  return LCE_OK;
}

// the planes cp[0..ncp) of every slab, once its neighbours' streams have
// recorded ev_pass; then each stream waits for its neighbours' copies before
// a later pass may overwrite the planes they read
int slab_exchange(lce_slabs* S, const PlaneCopy* cp, int ncp) {
  const int n = (int)S->slab.size();
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    DeviceScope ds_(c->device);
    SCK(cudaStreamWaitEvent(c->stream, S->ev_pass[(k + n - 1) % n], 0));
    SCK(cudaStreamWaitEvent(c->stream, S->ev_pass[(k + 1) % n], 0));
    for (int i = 0; i < ncp; ++i)
      if (int rc = slab_copy_plane(c, S->slab[(k + n + cp[i].dk) % n], cp[i], S->nxy)) return rc;
    SCK(cudaEventRecord(S->ev_copy[k], c->stream));
  }
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    DeviceScope ds_(c->device);
    SCK(cudaStreamWaitEvent(c->stream, S->ev_copy[(k + n - 1) % n], 0));
    SCK(cudaStreamWaitEvent(c->stream, S->ev_copy[(k + 1) % n], 0));
  }
  return LCE_OK;
}

// the measured quantities of the whole lattice from the slabs' summed
// per-slot totals: the formulas of the finalize kernel (f/meas1.f inputs,
// f/ahiggs2.f:142-147, f/agauge.f:195-200, f/agauge1.f:227-232)
// delta: the whole lattice's ahiggs1 step, adapted as the finalize kernel
// adapts it (f/ahiggs1.f:113-123, in the fields' precision) from the whole
// lattice's acceptance
void slab_meas(const std::vector<double>& tot, const FinalizeArgs& f, double V, lce_meas* m, double* delta) {
  double h[kNQ] = {0, 0, 0, 0}, l[kNQ] = {0, 0, 0, 0};
  for (int i = 0; i < f.nslots; ++i) {
    const double* t = tot.data() + (size_t)i * kNQ;
    const int kind = f.kinds[i] & 0x7f;
    const bool end = (f.kinds[i] & kKindEnd) != 0;
    double* acc = kind <= kHiggsMetro ? h : l;
    for (int q = 0; q < kNQ; ++q) acc[q] += t[q];
    if (!end) continue;
    if (kind == kHiggsHB || kind == kHiggsOR || kind == kHiggsMetro) {
      m->a2 = h[1] / V;
      m->a4 = h[2] / V;
      m->akin = h[3] / (6.0 * V);
      if (kind == kHiggsHB) m->acc_hb = h[0] / V;
      if (kind == kHiggsOR) m->acc_or = h[0] / V;
      if (kind == kHiggsMetro) {
        if (f.single) {
          const float a = (float)h[0] / (float)V;
          float d = (float)*delta;
          if (fabsf(a - 0.5f) > 0.1f) d = (a > 0.5f) ? 1.1131241f * d : 0.8989669f * d;
          m->acc_metro = a;
          *delta = d;
        } else {
          const double a = h[0] / V;
          double d = *delta;
          if (fabs(a - 0.5) > 0.1) d = (a > 0.5) ? 1.1131241 * d : 0.8989669 * d;
          m->acc_metro = a;
          *delta = d;
        }
      }
    } else if (kind == kLinkHB) {
      m->plaq = l[2] / (12.0 * V);
      m->acc_gauge = (l[0] / (3.0 * V)) * (l[1] / (12.0 * V));
    } else if (kind == kLinkHB3) {
      m->plaq = l[2] / (12.0 * V);
      m->acc_gauge = (l[0] / (3.0 * V)) * (l[1] / (12.0 * V) / 3.0);
    } else if (kind == kLinkOR) {
      m->acc_link_or = l[0] / (3.0 * V);
    }
    for (int q = 0; q < kNQ; ++q) acc[q] = 0.0;
  }
}

int slab_sweep(lce_slabs* S, int measflag, lce_meas* m) {
  const int n = (int)S->slab.size();
  std::vector<Enq> q(n);
  const std::vector<unsigned char> routines = sweep_routines(S->slab[0]);
  for (int k = 0; k < n; ++k) enq_begin(S->slab[k], routines, measflag, true, kBlock, 1, 0, q[k]);
  for (size_t i = 0; i < q[0].passes.size(); ++i) {
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      if (int rc = enq_pass(c, q[k], i)) return slab_rc(c, rc);
      SCK(cudaEventRecord(S->ev_pass[k], c->stream));
    }
    const Pass& ps = q[0].passes[i];
    const int f = ps.kind <= kHiggsMetro ? -1 : ps.mu, nz = S->nz;
    const PlaneCopy cp[2] = {{-1, nz, 0, f, ps.eo, false}, {+1, 1, nz + 1, f, ps.eo, false}};
    if (int rc = slab_exchange(S, cp, 2)) return rc;
  }
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    DeviceScope ds_(c->device);
    if (int rc = enq_end(c, q[k])) return slab_rc(c, rc);
  }
  // per-slot totals (the slot count is known once the finalize is queued)
  std::vector<double> tot((size_t)q[0].f.nslots * kNQ, 0.0), t(tot.size());
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    DeviceScope ds_(c->device);
    if (int rc = status_check(c)) return slab_rc(c, rc);  // synchronises the slab's stream
    if (!t.empty()) {  // measured slots, and the Metropolis slots of every sweep
      SCK(cudaMemcpy(t.data(), c->totals_d, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (size_t e = 0; e < t.size(); ++e) tot[e] += t[e];
    }
  }
  lce_meas mm;
  std::memset(&mm, 0, sizeof(mm));
  slab_meas(tot, q[0].f, (double)S->L[0] * S->L[1] * S->L[2], &mm, &S->delta);
  mm.delta = S->delta;
  if (S->slab[0]->n_higgs_metro > 0) {
    // every slab's finalize adapted the step to its own acceptance: give them
    // the whole lattice's
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      SCK(cudaMemcpy(&c->cst_d[0].delta, &S->delta, sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  if (m) *m = mm;
  return LCE_OK;
}

// the overrelaxed Landau gauge fixing of f/landau_gauge.f:33-49 and
// f/or_gauge_fixing1.f on the slabs.  A half-step updates the U_z link below
// each site of a slab's first interior plane, which lives in the lower halo
// and belongs to slab k-1: after it that link goes back to slab k-1 (its
// plane nz), and slab k-1's plane nz of the updated parity comes forward into
// slab k's halo (the next half-step's U_f(x - z, z)).  Nothing else crosses
// a slab boundary.  Theta (the whole lattice's odd sites, before their
// update) is summed per slab, combined on slab 0's device, and the count and
// stop decision copied to every slab's chain state, all ordered by events: no host
// round trip inside a batch of iterations.
// it_flags >= 0: the half-steps of f/it_gauge_fixing.f with these flags
// (LCE_ITGF_*) instead of the overrelaxed ones
template <typename R>
int slab_gf_iterations(lce_slabs* S, int batch, int track, int it_flags = -1) {
  const int n = (int)S->slab.size(), nz = S->nz;
  lce_ctx* c0 = S->slab[0];
  const size_t off = offsetof(ChainState, gf_theta), len = offsetof(ChainState, gf_pad) - off;
  const double nh_all = (double)S->nxy * S->L[2];
  for (int it = 0; it < batch; ++it) {
    for (int pg = 0; pg < 2; ++pg) {
      for (int k = 0; k < n; ++k) {
        lce_ctx* c = S->slab[k];
        DeviceScope ds_(c->device);
        if (it_flags >= 0)
          launch_it_half<R>(c->ch_d, c->cst_d, pg ^ c->eo_flip, pg, c->scratch_d, c->ch[0].nh, c->s_lo, it_flags,
                            c->stream);
        else
          launch_gf_half<R>(c->ch_d, c->cst_d, pg ^ c->eo_flip, pg, c->scratch_d, c->ch[0].nh, c->s_lo, track,
                            c->stream);
        SCK(cudaGetLastError());
        SCK(cudaEventRecord(S->ev_pass[k], c->stream));
      }
      const PlaneCopy cp[2] = {{+1, 0, nz, 2, pg ^ 1, true}, {-1, nz, 0, 2, pg, true}};
      if (int rc = slab_exchange(S, cp, 2)) return rc;
    }
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      const int nb = ceil_div(c->ch[0].nh - 2 * c->s_lo, kBlock);
      launch_sum_partials(c->scratch_d, nb, 1, c->scratch_d + nb, c->stream);
      SCK(cudaGetLastError());
      if (c->device == c0->device)
        SCK(cudaMemcpyAsync(S->g_d + k, c->scratch_d + nb, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      else
        SCK(cudaMemcpyPeerAsync(S->g_d + k, c0->device, c->scratch_d + nb, c->device, sizeof(double), c->stream));
      SCK(cudaEventRecord(S->ev_sum[k], c->stream));
    }
    {
      DeviceScope ds_(c0->device);
      for (int k = 1; k < n; ++k) SCK(cudaStreamWaitEvent(c0->stream, S->ev_sum[k], 0));
      launch_gf_check_slabs(c0->ch_d, c0->cst_d, S->g_d, n, nh_all, c0->stream);
      SCK(cudaGetLastError());
      SCK(cudaEventRecord(S->ev_chk, c0->stream));
    }
    for (int k = 1; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      SCK(cudaStreamWaitEvent(c->stream, S->ev_chk, 0));
      char* dst = (char*)c->cst_d + off;
      const char* src = (const char*)c0->cst_d + off;
      if (c->device == c0->device) SCK(cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToDevice, c->stream));
      else SCK(cudaMemcpyPeerAsync(dst, c->device, src, c0->device, len, c->stream));
    }
  }
  return LCE_OK;
}

// One batch of Fourier-accelerated iterations on the slabs (the stages of
// launch_fa_slab_stage): (a) every slab: Delta and the x transforms of its
// interior lines into the whole lattice's buffer on the first slab's
// device, theta summed per slab and copied there; (b) the first slab: the
// check (theta of the whole lattice, iteration count, done flag, step) and
// the y and z transforms (cg: with the momentum-space sums and beta);
// (c) every slab: the chain state (cg: and the CG state) from the first, the
// inverse x transforms and g (cg: the direction) at its interior sites;
// (d) g of the plane above each slab into its upper halo -- cg: the
// direction's plane instead, then every slab's line derivatives summed per
// slab and gathered on the first slab, the step there, the CG state back to
// every slab and g = exp(alpha X) at every local site; (e) every slab: g
// applied at its interior sites (links, A_f, G); (f) the U_z links of the
// plane below each slab into its lower halo.  Slabs write and read only the
// lines of their own planes in the buffer; the transforms of (b) run
// between the two.
template <typename R>
int slab_fa_iterations(lce_slabs* S, int batch, bool cg) {
  const int n = (int)S->slab.size(), nz = S->nz;
  lce_ctx* c0 = S->slab[0];
  const int Lg[3] = {S->L[0], S->L[1], S->L[2]};
  const double nh_all = (double)S->nxy * S->L[2];
  const size_t off = offsetof(ChainState, gf_theta), len = sizeof(ChainState) - off;
  const FaSlabCg* cgw = cg ? &S->cgw : nullptr;
  // the CG state of the first slab's device into every slab's buffer
  auto cg_state_to_slabs = [&]() -> int {
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      if (k > 0) SCK(cudaStreamWaitEvent(c->stream, S->ev_chk, 0));
      void* dst = fa_cg_state(c->fa_d, fa_vcap(c));
      if (c->device == c0->device)
        SCK(cudaMemcpyAsync(dst, S->cgw.cg, fa_cg_state_bytes(), cudaMemcpyDeviceToDevice, c->stream));
      else
        SCK(cudaMemcpyPeerAsync(dst, c->device, S->cgw.cg, c0->device, fa_cg_state_bytes(), c->stream));
    }
    return LCE_OK;
  };
  for (int it = 0; it < batch; ++it) {
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      const int nb = launch_fa_slab_stage<R>(0, c->ch_d, c->ch[0], c->cst_d, S->fft_d, c->fa_d, fa_vcap(c),
                                             c->scratch_d, Lg, 1, nz, k * nz, c->s_lo, c->stream);
      const std::string fe = fa_take_error();
      if (!fe.empty()) return slabs_fail(LCE_ERR_CUDA, "slabs Fourier fixing: " + fe);
      launch_sum_partials(c->scratch_d, nb, 1, c->scratch_d + nb, c->stream);
      SCK(cudaGetLastError());
      if (c->device == c0->device)
        SCK(cudaMemcpyAsync(S->g_d + k, c->scratch_d + nb, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      else
        SCK(cudaMemcpyPeerAsync(S->g_d + k, c0->device, c->scratch_d + nb, c->device, sizeof(double), c->stream));
      SCK(cudaEventRecord(S->ev_sum[k], c->stream));
    }
    {
      DeviceScope ds_(c0->device);
      for (int k = 1; k < n; ++k) SCK(cudaStreamWaitEvent(c0->stream, S->ev_sum[k], 0));
      launch_gf_check_slabs(c0->ch_d, c0->cst_d, S->g_d, n, nh_all, c0->stream, cg ? 2 : 1);
      launch_fa_slab_stage<R>(1, c0->ch_d, c0->ch[0], c0->cst_d, S->fft_d, c0->fa_d, fa_vcap(c0), nullptr, Lg, 1, nz,
                              0, c0->s_lo, c0->stream, cgw);
      const std::string fe = fa_take_error();
      if (!fe.empty()) return slabs_fail(LCE_ERR_CUDA, "slabs Fourier fixing: " + fe);
      SCK(cudaGetLastError());
      SCK(cudaEventRecord(S->ev_chk, c0->stream));
    }
    if (cg) {
      if (int rc = cg_state_to_slabs()) return rc;
    }
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      if (k > 0) {
        SCK(cudaStreamWaitEvent(c->stream, S->ev_chk, 0));
        char* dst = (char*)c->cst_d + off;
        const char* src = (const char*)c0->cst_d + off;
        if (c->device == c0->device) SCK(cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToDevice, c->stream));
        else SCK(cudaMemcpyPeerAsync(dst, c->device, src, c0->device, len, c->stream));
      }
      launch_fa_slab_stage<R>(2, c->ch_d, c->ch[0], c->cst_d, S->fft_d, c->fa_d, fa_vcap(c), nullptr, Lg, 1, nz,
                              k * nz, c->s_lo, c->stream, cgw);
      const std::string fe = fa_take_error();
      if (!fe.empty()) return slabs_fail(LCE_ERR_CUDA, "slabs Fourier fixing: " + fe);
      SCK(cudaGetLastError());
      SCK(cudaEventRecord(S->ev_pass[k], c->stream));
    }
    if (cg) {
      const PlaneCopy dcp[2] = {{+1, 1, nz + 1, 5, 0, false}, {+1, 1, nz + 1, 5, 1, false}};
      if (int rc = slab_exchange(S, dcp, 2)) return rc;
      for (int k = 0; k < n; ++k) {
        lce_ctx* c = S->slab[k];
        DeviceScope ds_(c->device);
        const int nb = launch_fa_slab_stage<R>(4, c->ch_d, c->ch[0], c->cst_d, S->fft_d, c->fa_d, fa_vcap(c),
                                               nullptr, Lg, 1, nz, k * nz, c->s_lo, c->stream, cgw);
        // the slab's triple into its scratch, then to the first slab's device
        launch_sum_partials(fa_cgpart_ptr(c->fa_d, fa_vcap(c)), nb, 3, c->scratch_d, c->stream);
        SCK(cudaGetLastError());
        double* dst = S->cgw.tri + 3 * (size_t)k;
        if (c->device == c0->device)
          SCK(cudaMemcpyAsync(dst, c->scratch_d, 3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        else
          SCK(cudaMemcpyPeerAsync(dst, c0->device, c->scratch_d, c->device, 3 * sizeof(double), c->stream));
        SCK(cudaEventRecord(S->ev_sum[k], c->stream));
      }
      {
        DeviceScope ds_(c0->device);
        for (int k = 1; k < n; ++k) SCK(cudaStreamWaitEvent(c0->stream, S->ev_sum[k], 0));
        launch_fa_slab_stage<R>(5, c0->ch_d, c0->ch[0], c0->cst_d, S->fft_d, c0->fa_d, fa_vcap(c0), nullptr, Lg, 1,
                                nz, 0, c0->s_lo, c0->stream, cgw);
        SCK(cudaGetLastError());
        SCK(cudaEventRecord(S->ev_chk, c0->stream));
      }
      if (int rc = cg_state_to_slabs()) return rc;
      for (int k = 0; k < n; ++k) {
        lce_ctx* c = S->slab[k];
        DeviceScope ds_(c->device);
        launch_fa_slab_stage<R>(6, c->ch_d, c->ch[0], c->cst_d, S->fft_d, c->fa_d, fa_vcap(c), nullptr, Lg, 1, nz,
                                k * nz, c->s_lo, c->stream, cgw);
        SCK(cudaGetLastError());
      }
    } else {
      const PlaneCopy gcp[2] = {{+1, 1, nz + 1, 4, 0, false}, {+1, 1, nz + 1, 4, 1, false}};
      if (int rc = slab_exchange(S, gcp, 2)) return rc;
    }
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      launch_fa_slab_stage<R>(3, c->ch_d, c->ch[0], c->cst_d, S->fft_d, c->fa_d, fa_vcap(c), nullptr, Lg, 1, nz,
                              k * nz, c->s_lo, c->stream);
      SCK(cudaGetLastError());
      SCK(cudaEventRecord(S->ev_pass[k], c->stream));
    }
    const PlaneCopy ucp[2] = {{-1, nz, 0, 2, 0, true}, {-1, nz, 0, 2, 1, true}};
    if (int rc = slab_exchange(S, ucp, 2)) return rc;
  }
  return LCE_OK;
}

// The start of a gauge fixing on the slabs.  start < 0: the reference's
// fixing from U (no transform kept); otherwise a tracked fixing (G
// accumulated as in lce_landau_gauge_from) from G = 1 (LCE_GF_START_IDENTITY)
// or from the transform the slabs hold (LCE_GF_START_TRANSFORM: the G planes
// next to every slab boundary are exchanged into the halos, then U_f = G U
// G^+ and A_f = G A G^+ on every plane of every slab -- a slab's halo planes
// get the values its neighbours compute for them, so the start equals the
// undecomposed one bit for bit)
int slab_gf_start(lce_slabs* S, int start) {
  const int n = (int)S->slab.size(), nz = S->nz;
  if (start == LCE_GF_START_TRANSFORM) {
    for (int k = 0; k < n; ++k) {
      lce_ctx* c = S->slab[k];
      DeviceScope ds_(c->device);
      SCK(cudaEventRecord(S->ev_pass[k], c->stream));
    }
    const PlaneCopy cp[4] = {{-1, nz, 0, 3, 0, false}, {-1, nz, 0, 3, 1, false},
                             {+1, 1, nz + 1, 3, 0, false}, {+1, 1, nz + 1, 3, 1, false}};
    if (int rc = slab_exchange(S, cp, 4)) return rc;
  }
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    DeviceScope ds_(c->device);
    const ChainDev& ch = c->ch[0];
    if (start == LCE_GF_START_TRANSFORM) {
      if (c->prec == LCE_PREC_F64) launch_gauge_apply<double>(c->ch_d, ch.nh, c->stream);
      else launch_gauge_apply<float>(c->ch_d, ch.nh, c->stream);
      SCK(cudaGetLastError());
    } else {
      const size_t ub = (size_t)6 * ch.nh * link_bytes(c->prec), ab = (size_t)6 * ch.nh * real_bytes(c->prec);
      SCK(cudaMemcpyAsync(ch.uf, ch.u, ub, cudaMemcpyDeviceToDevice, c->stream));
      SCK(cudaMemcpyAsync(ch.af, ch.a, ab, cudaMemcpyDeviceToDevice, c->stream));
      if (start == LCE_GF_START_IDENTITY) {
        if (c->prec == LCE_PREC_F64) launch_transform_identity<double>(ch.g, ch.nh, c->stream);
        else launch_transform_identity<float>(ch.g, ch.nh, c->stream);
        SCK(cudaGetLastError());
      }
    }
  }
  return LCE_OK;
}

// every slab's chain state for a fixing: not done, no iterations, the cap;
// limit and step: the Fourier iteration's stopping theta and step (< 0: kept)
int slab_gf_state(lce_slabs* S, int cap, double limit = -1.0, double step = -1.0) {
  for (lce_ctx* c : S->slab) {
    DeviceScope ds_(c->device);
    ChainState cs;
    SCK(cudaMemcpyAsync(&cs, c->cst_d, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
    SCK(cudaStreamSynchronize(c->stream));
    cs.gf_done = 0;
    cs.gf_iters = 0;
    cs.gf_cap = cap;
    cs.gf_theta = 1.0e4;
    if (limit >= 0.0) cs.gf_limit = limit;
    if (step >= 0.0) cs.gf_step = step;
    SCK(cudaMemcpyAsync(c->cst_d, &cs, sizeof(cs), cudaMemcpyHostToDevice, c->stream));
    SCK(cudaStreamSynchronize(c->stream));
  }
  return LCE_OK;
}

// batches of iterations (overrelaxed, or Fourier-accelerated with fourier)
// until the first slab's chain state says done; its final state in cs
int slab_gf_run(lce_slabs* S, int track, bool fourier, ChainState& cs, int it_flags = -1, bool cg = false) {
  lce_ctx* c0 = S->slab[0];
  std::memset(&cs, 0, sizeof(cs));
  int batch = fourier ? 4 : 8;
  while (true) {
    int rc;
    if (fourier)
      rc = S->prec == LCE_PREC_F64 ? slab_fa_iterations<double>(S, batch, cg)
                                   : slab_fa_iterations<float>(S, batch, cg);
    else
      rc = S->prec == LCE_PREC_F64 ? slab_gf_iterations<double>(S, batch, track, it_flags)
                                   : slab_gf_iterations<float>(S, batch, track, it_flags);
    if (rc) return rc;
    const int before = cs.gf_iters;
    {
      DeviceScope ds_(c0->device);
      SCK(cudaMemcpyAsync(&cs, c0->cst_d, sizeof(cs), cudaMemcpyDeviceToHost, c0->stream));
      SCK(cudaStreamSynchronize(c0->stream));
    }
    if (cs.gf_done) break;
    if (cs.gf_iters <= before) return slabs_fail(LCE_ERR_CUDA, "slabs gauge fixing: a batch made no progress");
    if (batch < 64) batch *= 2;
  }
  for (lce_ctx* c : S->slab) {
    DeviceScope ds_(c->device);
    SCK(cudaStreamSynchronize(c->stream));
  }
  return LCE_OK;
}

int slab_landau_gauge(lce_slabs* S, double* theta, int* iters, int max_iters, int start = -1) {
  lce_ctx* c0 = S->slab[0];
  const int cap = max_iters > 0 ? max_iters : 1000000;
  if (int rc = slab_gf_start(S, start)) return rc;
  if (int rc = slab_gf_state(S, cap)) return rc;
  ChainState cs;
  if (int rc = slab_gf_run(S, start >= 0 ? 1 : 0, false, cs)) return rc;
  if (theta) *theta = cs.gf_theta;
  if (iters) *iters = cs.gf_iters;
  if (!std::isfinite(cs.gf_theta)) return slabs_fail(LCE_ERR_NAN, "slabs gauge fixing: theta is not finite");
  if (cs.gf_theta > c0->ch[0].limit_or)
    return slabs_fail(LCE_ERR_GF_NOT_CONVERGED, "slabs gauge fixing: iteration cap reached");
  return LCE_OK;
}

// lce_landau_gauge_fourier on the slabs: Fourier-accelerated iterations to
// theta_switch, then the overrelaxed iteration to limit_or, tracking G
int slab_fourier_fix(lce_slabs* S, int start, double step, double theta_switch, double* theta, int* iters_f,
                     int* iters_p, int max_iters, bool cg = false) {
  lce_ctx* c0 = S->slab[0];
  const double limit = c0->ch[0].limit_or;
  if (!(step > 0.0)) step = 1.0;
  if (!(theta_switch > 0.0)) theta_switch = limit;
  for (int d = 0; d < 3; ++d) {
    int lg = 0;
    while ((1 << lg) < S->L[d]) ++lg;
    if ((1 << lg) != S->L[d] || lg < 1 || S->L[d] > 1024)
      return slabs_fail(LCE_ERR_UNSUPPORTED, "slabs Fourier fixing: extents must be powers of two up to 1024");
  }
  for (lce_ctx* c : S->slab) {
    DeviceScope ds_(c->device);
    if (int rc = fa_buffers(c)) return slab_rc(c, rc);
  }
  if (!S->fft_d) {
    DeviceScope ds_(c0->device);
    const size_t V = (size_t)S->L[0] * S->L[1] * S->L[2];
    if (cudaMalloc(&S->fft_d, 2 * V * 2 * sizeof(float)) != cudaSuccess) {
      S->fft_d = nullptr;
      cudaGetLastError();
      return slabs_fail(LCE_ERR_NOMEM, "slabs Fourier fixing: the whole lattice's transform buffer");
    }
  }
  if (cg && !S->cg_d) {
    // the CG state (256 bytes), F of this and the previous iteration, the z
    // transform's per-block pairs and one line triple per slab
    DeviceScope ds_(c0->device);
    const size_t V = (size_t)S->L[0] * S->L[1] * S->L[2];
    int lz = 0;
    while ((1 << lz) < S->L[2]) ++lz;
    const size_t nbz = (V / S->L[2] + (4096 >> lz) - 1) / (4096 >> lz);
    const size_t prev_b = 4 * V * 2 * sizeof(float), pairs_n = 2 * 2 * nbz, tri_n = 3 * S->slab.size();
    if (cudaMalloc(&S->cg_d, 256 + prev_b + (pairs_n + tri_n) * sizeof(double)) != cudaSuccess) {
      S->cg_d = nullptr;
      cudaGetLastError();
      return slabs_fail(LCE_ERR_NOMEM, "slabs Fourier CG fixing: the whole lattice's CG buffers");
    }
    char* b = static_cast<char*>(S->cg_d);
    S->cgw.cg = b;
    S->cgw.prev = b + 256;
    S->cgw.pairs = reinterpret_cast<double*>(b + 256 + prev_b);
    S->cgw.tri = S->cgw.pairs + pairs_n;
    S->cgw.nslabs = (int)S->slab.size();
    S->cgw.nh_all = (double)S->nxy * S->L[2];
  }
  const int cap = max_iters > 0 ? max_iters : 1000000;
  if (int rc = slab_gf_start(S, start)) return rc;
  if (int rc = slab_gf_state(S, cap, theta_switch, step)) return rc;
  if (cg) {
    DeviceScope ds_(c0->device);
    fa_cg_reset_state(S->cgw.cg, c0->stream);
    SCK(cudaGetLastError());
  }
  ChainState cs;
  if (int rc = slab_gf_run(S, 1, true, cs, -1, cg)) return rc;
  if (iters_f) *iters_f = cs.gf_iters;
  if (iters_p) *iters_p = 0;
  if (theta) *theta = cs.gf_theta;
  if (!std::isfinite(cs.gf_theta)) return slabs_fail(LCE_ERR_NAN, "slabs Fourier fixing: theta is not finite");
  if (cs.gf_theta <= limit) return LCE_OK;
  const int it_fa = cs.gf_iters;
  if (it_fa >= cap) return slabs_fail(LCE_ERR_GF_NOT_CONVERGED, "slabs Fourier fixing: iteration cap reached");
  // the overrelaxed iteration from theta_switch to limit_or
  if (int rc = slab_gf_state(S, cap - it_fa)) return rc;
  if (int rc = slab_gf_run(S, 1, false, cs)) return rc;
  if (iters_p) *iters_p = cs.gf_iters;
  if (theta) *theta = cs.gf_theta;
  if (!std::isfinite(cs.gf_theta)) return slabs_fail(LCE_ERR_NAN, "slabs gauge fixing: theta is not finite");
  if (cs.gf_theta > limit) return slabs_fail(LCE_ERR_GF_NOT_CONVERGED, "slabs gauge fixing: iteration cap reached");
  return LCE_OK;
}

// the z-slice sums of every slab's interior planes (the slice_sums kernel on
// each slab's own device), gathered into the whole lattice's slices on slab
// 0's device, and the correlators of lce_correlator formed there; h
// receives the 7 L3 + 5 values of the correlator kernel's output
int slab_slices(lce_slabs* S, std::vector<double>& h) {
  const int n = (int)S->slab.size(), nz = S->nz, L3 = S->L[2];
  lce_ctx* c0 = S->slab[0];
  double* slices = S->g_d + n;
  double* out = slices + (size_t)14 * L3;
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    DeviceScope ds_(c->device);
    if (S->prec == LCE_PREC_F64) launch_slice_sums<double>(c->ch_d, nz + 2, c->scratch_d, c->stream);
    else launch_slice_sums<float>(c->ch_d, nz + 2, c->scratch_d, c->stream);
    SCK(cudaGetLastError());
    const size_t bytes = (size_t)14 * nz * sizeof(double);
    double* dst = slices + (size_t)14 * k * nz;
    if (c->device == c0->device)
      SCK(cudaMemcpyAsync(dst, c->scratch_d + 14, bytes, cudaMemcpyDeviceToDevice, c->stream));
    else
      SCK(cudaMemcpyPeerAsync(dst, c0->device, c->scratch_d + 14, c->device, bytes, c->stream));
    SCK(cudaEventRecord(S->ev_sum[k], c->stream));
  }
  DeviceScope ds_(c0->device);
  for (int k = 1; k < n; ++k) SCK(cudaStreamWaitEvent(c0->stream, S->ev_sum[k], 0));
  launch_correlators(slices, S->L[0], S->L[1], L3, out, c0->stream);
  SCK(cudaGetLastError());
  h.assign((size_t)7 * L3 + 5, 0.0);
  SCK(cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c0->stream));
  SCK(cudaStreamSynchronize(c0->stream));
  return LCE_OK;
}

// whole-lattice arrays (reference order: u[mu][eo][site < ld][4],
// a[eo][site < ld][3]) <-> each slab's planes, halos included on the way in;
// which: the fields or (downloads only) the gauge-fixed copies
template <typename T>
int slabs_copy(lce_slabs* S, T* u, T* a, long ld, bool in, int which = LCE_FIELDS) {
  const int n = (int)S->slab.size(), nz = S->nz, nxy = S->nxy, L3 = S->L[2];
  const long nhl = (long)(nz + 2) * nxy;
  std::vector<T> ul((size_t)6 * nhl * 4), al((size_t)2 * nhl * 3);
  for (int k = 0; k < n; ++k) {
    lce_ctx* c = S->slab[k];
    const int z0 = k * nz;
    if (!in) {
      int rc = std::is_same<T, double>::value
                   ? lce_download_f64(c, 0, which, (double*)ul.data(), (double*)al.data(), nhl)
                   : lce_download(c, 0, which, (float*)ul.data(), (float*)al.data(), nhl);
      if (rc) return slab_rc(c, rc);
    }
    for (int zl = in ? 0 : 1; zl <= (in ? nz + 1 : nz); ++zl) {
      const int zg = (z0 - 1 + zl + L3) % L3;
      for (int pl = 0; pl < 2; ++pl) {
        const int pg = pl ^ c->eo_flip;
        for (int mu = 0; mu < 3; ++mu) {
          T* loc = &ul[(((size_t)mu * 2 + pl) * nhl + (size_t)zl * nxy) * 4];
          T* glo = &u[(((size_t)mu * 2 + pg) * ld + (size_t)zg * nxy) * 4];
          if (in) std::memcpy(loc, glo, sizeof(T) * 4 * nxy);
          else std::memcpy(glo, loc, sizeof(T) * 4 * nxy);
        }
        T* loc = &al[((size_t)pl * nhl + (size_t)zl * nxy) * 3];
        T* glo = &a[((size_t)pg * ld + (size_t)zg * nxy) * 3];
        if (in) std::memcpy(loc, glo, sizeof(T) * 3 * nxy);
        else std::memcpy(glo, loc, sizeof(T) * 3 * nxy);
      }
    }
    if (in) {
      int rc = std::is_same<T, double>::value
                   ? lce_upload_f64(c, 0, LCE_FIELDS, (const double*)ul.data(), (const double*)al.data(), nhl)
                   : lce_upload(c, 0, LCE_FIELDS, (const float*)ul.data(), (const float*)al.data(), nhl);
      if (rc) return slab_rc(c, rc);
    }
  }
  return LCE_OK;
}

}  // namespace

extern "C" {

const char* lce_version(void) { return "lceqcd_b200 1.0 (sm_100a)"; }

const char* lce_strerror(int s) {
  switch (s) {
    case LCE_OK: return "ok";
    case LCE_ERR_INVALID: return "invalid argument";
    case LCE_ERR_CUDA: return "CUDA error";
    case LCE_ERR_GF_NOT_CONVERGED: return "gauge fixing did not converge";
    case LCE_ERR_STREAM: return "validation uniform stream exhausted";
    case LCE_ERR_NAN: return "non-finite value";
    case LCE_ERR_NOMEM: return "out of device memory";
    case LCE_ERR_UNSUPPORTED: return "unsupported for this context";
    default: return "unknown status";
  }
}

const char* lce_last_error(lce_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

void lce_default_params(lce_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->L[0] = p->L[1] = p->L[2] = 16;
  p->beta = 9.0;
  p->x = 0.1;
  p->y = 0.5;
  p->lambda = 1.8;
  p->alpha = 1.0;
  p->limit_or = 1.0e-9;
  p->imode = 0;
  p->precision = LCE_PREC_F32;
  p->rng = LCE_RNG_PHILOX;
  p->seed = 12345;
  p->device = 0;
  p->delta0 = 1.0;
  p->gf_angle = LCE_GF_ATAN2;
  p->sweep_mode = LCE_SWEEP_AUTO;
  p->agauge_hits = 1;
}

int lce_couplings(const lce_params* p, double out[3]) {
  if (!p || !out) return LCE_ERR_INVALID;
  if (p->precision == LCE_PREC_F32) couplings_t<float>(p->beta, p->x, p->y, out);
  else couplings_t<double>(p->beta, p->x, p->y, out);
  return LCE_OK;
}

int lce_geometry_tables(int L1, int L2, int L3, int* siteup, int* sitedn) {
  if (L1 < 2 || L2 < 2 || L3 < 2 || (L1 | L2 | L3) & 1 || !siteup || !sitedn) return LCE_ERR_INVALID;
  const int hx = L1 / 2, nxy = L1 * L2 / 2, nh = nxy * L3;
  const FastDiv dhx = make_fastdiv(hx), dnxy = make_fastdiv(nxy);
  const int L[3] = {L1, L2, L3};
  for (int eo = 0; eo < 2; ++eo)
    for (int s = 0; s < nh; ++s) {
      Coord X = site_coord(eo, s, hx, nxy, dhx, dnxy);
      for (int mu = 0; mu < 3; ++mu) {
        int cu[3] = {X.x, X.y, X.z}, cd[3] = {X.x, X.y, X.z};
        cu[mu] = wrap(cu[mu] + 1, L[mu]);
        cd[mu] = wrap(cd[mu] - 1, L[mu]);
        siteup[((size_t)eo * 3 + mu) * nh + s] = site_index(cu[0], cu[1], cu[2], hx, nxy);
        sitedn[((size_t)eo * 3 + mu) * nh + s] = site_index(cd[0], cd[1], cd[2], hx, nxy);
      }
    }
  return LCE_OK;
}

lce_ctx* lce_create(const lce_params* p) {
  DeviceScope ds_(p ? p->device : -1);
  return create_impl(p, 1);
}
lce_ctx* lce_create_batch(const lce_params* p, int nchains) {
  DeviceScope ds_(p && nchains > 0 ? p->device : -1);
  return create_impl(p, nchains);
}

void lce_destroy(lce_ctx* c) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->sweep_graphs)
    if (kv.second) cudaGraphExecDestroy(kv.second);
  for (auto& kv : c->gf_exec) cudaGraphExecDestroy(kv.second);
  for (auto& kv : c->fa_exec) cudaGraphExecDestroy(kv.second);
  void* ptrs[] = {c->ch_d, c->tiles_d[0], c->tiles_d[1], c->tiles_d[2], c->tiles_d[3], c->st_d, c->cst_d, c->meas_d, c->part_d, c->totals_d,
                  c->scratch_d, c->fields_d, c->stream_d, c->staging_d, c->flush_d, c->bar_d,
                  c->gsave_d, c->fa_d, c->chunks_begin_d[0], c->chunks_begin_d[1], c->chunks_begin_d[2],
                  c->chunks_begin_d[3],
                  c->chunks_d, c->async_d};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->join_ev) cudaEventDestroy(c->join_ev);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->copy) {
    cudaStreamSynchronize(c->copy);
    cudaStreamDestroy(c->copy);
  }
  for (int k = 0; k < 2; ++k) {
    if (c->staged_ev[k]) cudaEventDestroy(c->staged_ev[k]);
    if (c->free_ev[k]) cudaEventDestroy(c->free_ev[k]);
  }
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

int lce_nchains(lce_ctx* c) { return c ? c->nchains : LCE_ERR_INVALID; }

int lce_get_extents(lce_ctx* c, int chain, int L[3]) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !L || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  L[0] = c->ch[chain].L1;
  L[1] = c->ch[chain].L2;
  L[2] = c->ch[chain].L3;
  return LCE_OK;
}

int lce_set_stream(lce_ctx* c, void* s) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  c->stream = s ? (cudaStream_t)s : c->own;
  return LCE_OK;
}

int lce_synchronize(lce_ctx* c) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  CK(cudaStreamSynchronize(c->stream));
  return status_check(c);
}

int lce_upload(lce_ctx* c, int chain, int which, const float* u, const float* a, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  return upload_t<float>(c, chain, which, u, a, ld);
}
// Asynchronous uploads in two steps.  lce_upload_stage: the host-to-device
// copies run on a copy stream into one of two staging slots (after the
// previous upload through that slot has been applied).  lce_upload_apply: the
// context stream waits for the oldest staged upload and copies it into the
// fields (links: one device copy; A: the layout kernel of lce_upload).  With
// two slots a client can stage the upload of step k+2 while step k+1's is
// applied behind step k's sweeps, so the copy engine never waits for the
// client.
int lce_upload_stage(lce_ctx* c, int chain, int which, const float* u, const float* a, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  if (c->prec != LCE_PREC_F32) return fail(c, LCE_ERR_UNSUPPORTED, "upload_stage: FP32 contexts only (lce_upload)");
  if (chain < 0 || chain >= c->nchains || (which != LCE_FIELDS && which != LCE_FIELDS_FIXED))
    return fail(c, LCE_ERR_INVALID, "upload_stage: bad chain or field selector");
  const ChainDev& ch = c->ch[chain];
  if (ld < ch.nh) return fail(c, LCE_ERR_INVALID, "upload_stage: ld smaller than L1*L2*L3/2");
  if (c->staged.size() >= 2) return fail(c, LCE_ERR_INVALID, "upload_stage: two staged uploads not yet applied");
  const size_t ulb = align256((size_t)6 * c->max_nh * 16);
  if (!c->copy) {
    CK(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
    c->async_slot = ulb + align256((size_t)6 * c->max_nh * sizeof(float));
    CK(cudaMalloc(&c->async_d, 2 * c->async_slot));
    for (int k = 0; k < 2; ++k) {
      CK(cudaEventCreateWithFlags(&c->staged_ev[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->free_ev[k], cudaEventDisableTiming));
      CK(cudaEventRecord(c->free_ev[k], c->stream));
    }
  }
  const int k = c->next_slot, nh = ch.nh;
  char* su = static_cast<char*>(c->async_d) + (size_t)k * c->async_slot;
  char* sa = su + ulb;
  CK(cudaStreamWaitEvent(c->copy, c->free_ev[k], 0));
  if (u) CK(cudaMemcpy2DAsync(su, (size_t)nh * 16, u, (size_t)ld * 16, (size_t)nh * 16, 6, cudaMemcpyHostToDevice, c->copy));
  if (a) CK(cudaMemcpy2DAsync(sa, (size_t)nh * 12, a, (size_t)ld * 12, (size_t)nh * 12, 2, cudaMemcpyHostToDevice, c->copy));
  CK(cudaEventRecord(c->staged_ev[k], c->copy));
  c->staged.push_back({k, chain, which | (u ? 2 : 0) | (a ? 4 : 0)});
  c->next_slot = 1 - k;
  return LCE_OK;
}

int lce_upload_apply(lce_ctx* c) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  if (c->staged.empty()) return fail(c, LCE_ERR_INVALID, "upload_apply: no staged upload");
  const std::array<int, 3> st = c->staged.front();
  c->staged.pop_front();
  const int k = st[0], which = st[2] & 1;
  const ChainDev& ch = c->ch[st[1]];
  const int nh = ch.nh;
  char* su = static_cast<char*>(c->async_d) + (size_t)k * c->async_slot;
  char* sa = su + align256((size_t)6 * c->max_nh * 16);
  CK(cudaStreamWaitEvent(c->stream, c->staged_ev[k], 0));
  if (st[2] & 2)
    CK(cudaMemcpyAsync(field_ptr(ch, which, true), su, (size_t)6 * nh * 16, cudaMemcpyDeviceToDevice, c->stream));
  if (st[2] & 4) launch_higgs_in<float, float>(reinterpret_cast<const float*>(sa), field_ptr(ch, which, false), nh, c->stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->free_ev[k], c->stream));
  return LCE_OK;
}

int lce_upload_async(lce_ctx* c, int chain, int which, const float* u, const float* a, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  if (!c->staged.empty()) return fail(c, LCE_ERR_INVALID, "upload_async: apply the staged uploads first");
  if (int rc = lce_upload_stage(c, chain, which, u, a, ld)) return rc;
  return lce_upload_apply(c);
}

int lce_upload_f64(lce_ctx* c, int chain, int which, const double* u, const double* a, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  return upload_t<double>(c, chain, which, u, a, ld);
}
int lce_download(lce_ctx* c, int chain, int which, float* u, float* a, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  return download_t<float>(c, chain, which, u, a, ld);
}
int lce_download_f64(lce_ctx* c, int chain, int which, double* u, double* a, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  return download_t<double>(c, chain, which, u, a, ld);
}

int lce_init_unit(lce_ctx* c, double a3) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  for (int i = 0; i < c->nchains; ++i) {
    if (c->prec == LCE_PREC_F64) launch_init_unit<double>(c->ch[i].u, c->ch[i].a, c->ch[i].nh, a3, c->stream);
    else launch_init_unit<float>(c->ch[i].u, c->ch[i].a, c->ch[i].nh, a3, c->stream);
  }
  CK(cudaGetLastError());
  return LCE_OK;
}

int lce_init_hot(lce_ctx* c, unsigned long long seed) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  for (int i = 0; i < c->nchains; ++i) {
    const unsigned long long k = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)i;
    const uint32_t k0 = (uint32_t)k, k1 = (uint32_t)(k >> 32);
    if (c->prec == LCE_PREC_F64) launch_init_hot<double>(c->ch[i].u, c->ch[i].a, c->ch[i].nh, k0, k1, c->stream);
    else launch_init_hot<float>(c->ch[i].u, c->ch[i].a, c->ch[i].nh, k0, k1, c->stream);
  }
  CK(cudaGetLastError());
  return LCE_OK;
}

int lce_set_rng_stream(lce_ctx* c, const double* u, size_t n) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || (!u && n)) return LCE_ERR_INVALID;
  if (c->rng != LCE_RNG_STREAM) return fail(c, LCE_ERR_UNSUPPORTED, "context was not created with LCE_RNG_STREAM");
  CK(cudaStreamSynchronize(c->stream));
  if (c->stream_d) CK(cudaFree(c->stream_d));
  c->stream_d = nullptr;
  c->stream_n = 0;
  if (n) {
    CK(cudaMalloc(&c->stream_d, n * sizeof(double)));
    CK(cudaMemcpy(c->stream_d, u, n * sizeof(double), cudaMemcpyHostToDevice));
  }
  c->stream_n = n;
  // graphs captured the old stream pointer
  for (auto& kv : c->sweep_graphs)
    if (kv.second) cudaGraphExecDestroy(kv.second);
  c->sweep_graphs.clear();
  unsigned long long z = 0;
  CK(cudaMemcpy(&c->st_d->stream_pos, &z, sizeof(z), cudaMemcpyHostToDevice));
  return LCE_OK;
}

int lce_get_rng_position(lce_ctx* c, unsigned long long* pass_ctr, unsigned long long* stream_pos) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  CtxState st;
  CK(cudaMemcpyAsync(&st, c->st_d, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (pass_ctr) *pass_ctr = st.pass_ctr;
  if (stream_pos) *stream_pos = st.stream_pos;
  return LCE_OK;
}

int lce_set_rng_position(lce_ctx* c, unsigned long long pass_ctr, unsigned long long stream_pos) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(&c->st_d->pass_ctr, &pass_ctr, sizeof(pass_ctr), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(&c->st_d->stream_pos, &stream_pos, sizeof(stream_pos), cudaMemcpyHostToDevice));
  return LCE_OK;
}

int lce_ahiggs1(lce_ctx* c, float* delta, int measflag, float* accept) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  if (delta) {
    // the step lives on the device; the caller's value is the one to use
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < c->nchains; ++i) {
      double d = *delta;
      CK(cudaMemcpy(&c->cst_d[i].delta, &d, sizeof(d), cudaMemcpyHostToDevice));
    }
  }
  float acc = 0;
  int rc = routine_call(c, kHiggsMetro, measflag, (accept || delta) ? &acc : nullptr, false);
  if (rc) return rc;
  if (accept) *accept = acc;
  if (delta) {
    double d;
    CK(cudaMemcpy(&d, &c->cst_d[0].delta, sizeof(d), cudaMemcpyDeviceToHost));
    *delta = (float)d;
  }
  return LCE_OK;
}

int lce_ahiggs2(lce_ctx* c, int measflag, float* accept) {
  DeviceScope ds_(c ? c->device : -1);
  return c ? routine_call(c, kHiggsHB, measflag, accept, false) : LCE_ERR_INVALID;
}
int lce_ahiggs3(lce_ctx* c, int measflag, float* accept) {
  DeviceScope ds_(c ? c->device : -1);
  return c ? routine_call(c, kHiggsOR, measflag, accept, false) : LCE_ERR_INVALID;
}
int lce_agauge(lce_ctx* c, int measflag, float* accept) {
  DeviceScope ds_(c ? c->device : -1);
  return c ? routine_call(c, kLinkHB, measflag, accept, false) : LCE_ERR_INVALID;
}
int lce_agauge1(lce_ctx* c, int measflag, float* accept) {
  DeviceScope ds_(c ? c->device : -1);
  return c ? routine_call(c, kLinkHB3, measflag, accept, false) : LCE_ERR_INVALID;
}
int lce_link_or(lce_ctx* c, int measflag, float* accept) {
  DeviceScope ds_(c ? c->device : -1);
  return c ? routine_call(c, kLinkOR, measflag, accept, false) : LCE_ERR_INVALID;
}

int lce_renorm(lce_ctx* c) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  for (int i = 0; i < c->nchains; ++i) {
    if (c->prec == LCE_PREC_F64) launch_renorm<double>(c->ch[i].u, (size_t)6 * c->ch[i].nh, c->stream);
    else launch_renorm<float>(c->ch[i].u, (size_t)6 * c->ch[i].nh, c->stream);
  }
  CK(cudaGetLastError());
  return LCE_OK;
}

int lce_sweeps(lce_ctx* c, int nsweeps, int measflag) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || nsweeps < 0) return LCE_ERR_INVALID;
  const int mf = measflag == 1 ? 1 : 0;
  int done = 0;
  // autotune: rotate through the candidates (sweep forms and tile shapes) on
  // real sweeps, one timed sweep at a time, until each has kTuneSamples
  // samples after a discarded first one; then keep the fastest by median.
  while (c->mode == LCE_SWEEP_AUTO && done < nsweeps) {
    int k = 0;
    for (int f = 1; f < (int)c->tune.size(); ++f)
      if (c->tune[f].ms.size() < c->tune[k].ms.size()) k = f;
    const TuneForm tf = c->tune[k];
    cudaGraphExec_t ex = nullptr;
    if (tf.form != LCE_SWEEP_DIRECT) {
      int rc = sweep_graph(c, tf.form, tf.bs, tf.spt, tf.occ, mf, &ex);
      if (rc) return rc;
      if (c->mode != LCE_SWEEP_AUTO) break;  // the persistent form was unavailable
    }
    CK(cudaEventRecord(c->ev0, c->stream));
    if (ex) CK(cudaGraphLaunch(ex, c->stream));
    else if (int rc = enqueue(c, sweep_routines(c), mf, true, nullptr, tf.bs, tf.spt, tf.occ)) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->tune[k].ms.push_back(ms);
    ++done;
    bool complete = true;
    for (const TuneForm& f : c->tune) complete = complete && f.ms.size() >= kTuneSamples + 1;
    if (complete) {
      int best = 0;
      float best_med = 0;
      for (int f = 0; f < (int)c->tune.size(); ++f) {
        std::vector<float> v(c->tune[f].ms.begin() + 1, c->tune[f].ms.end());
        std::sort(v.begin(), v.end());
        const float med = v[v.size() / 2];
        if (f == 0 || med < best_med) {
          best = f;
          best_med = med;
        }
      }
      c->mode = c->tune[best].form;
      c->tile_bs = c->tune[best].bs;
      c->tile_spt = c->tune[best].spt;
      c->tile_occ = c->tune[best].occ;
    }
  }
  if (done < nsweeps) {
    if (c->mode == LCE_SWEEP_DIRECT) {
      const std::vector<unsigned char> r = sweep_routines(c);
      for (int i = done; i < nsweeps; ++i)
        if (int rc = enqueue(c, r, mf, true)) return rc;
      return LCE_OK;
    }
    int i = done;
    if (nsweeps - i >= kSweepsPerGraph) {
      cudaGraphExec_t exm;
      if (int rc = sweep_graph(c, c->mode, c->tile_bs, c->tile_spt, c->tile_occ, mf, &exm, kSweepsPerGraph)) return rc;
      for (; nsweeps - i >= kSweepsPerGraph; i += kSweepsPerGraph) CK(cudaGraphLaunch(exm, c->stream));
    }
    if (i < nsweeps) {
      cudaGraphExec_t ex;
      if (int rc = sweep_graph(c, c->mode, c->tile_bs, c->tile_spt, c->tile_occ, mf, &ex)) return rc;
      for (; i < nsweeps; ++i) CK(cudaGraphLaunch(ex, c->stream));
    }
  }
  return LCE_OK;
}

int lce_get_sweep_mode(lce_ctx* c) { return c ? c->mode : LCE_ERR_INVALID; }

int lce_get_tile_shape(lce_ctx* c, int* threads, int* sites_per_thread, int* register_cap) {
  if (!c) return LCE_ERR_INVALID;
  const bool pers = c->mode == LCE_SWEEP_PERSISTENT;
  if (threads) *threads = pers ? kBlock : c->tile_bs;
  if (sites_per_thread) *sites_per_thread = pers ? 1 : c->tile_spt;
  if (register_cap) {
    // resident threads per SM the cap is set for: min_blocks_bs of the kernels
    const int bs = pers ? kBlock : c->tile_bs;
    const int blocks = std::max(1, (c->prec == LCE_PREC_F32 ? 4 : 3) * kBlock / bs);
    const int occ = pers || !c->tile_occ ? blocks * bs : c->tile_occ;
    *register_cap = std::min(255, (65536 / occ) & ~7);
  }
  return LCE_OK;
}

int lce_sweep(lce_ctx* c, int measflag, lce_meas* m) {
  DeviceScope ds_(c ? c->device : -1);
  int rc = lce_sweeps(c, 1, measflag);
  if (rc || !m) return rc;
  return lce_get_meas(c, 0, m);
}

int lce_get_meas(lce_ctx* c, int chain, lce_meas* m) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !m || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  CK(cudaMemcpyAsync(m, c->meas_d + chain, sizeof(*m), cudaMemcpyDeviceToHost, c->stream));
  int rc = status_check(c);
  if (rc) return rc;
  return LCE_OK;
}

int lce_get_meas_batch(lce_ctx* c, lce_meas* m) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !m) return LCE_ERR_INVALID;
  CK(cudaMemcpyAsync(m, c->meas_d, sizeof(lce_meas) * c->nchains, cudaMemcpyDeviceToHost, c->stream));
  return status_check(c);
}

int lce_landau_gauge(lce_ctx* c, int chain, double* theta, int* iters, int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  // f/landau_gauge.f:33-49 copy u -> u_f, a -> a_f
  const size_t ub = (size_t)6 * ch.nh * link_bytes(c->prec), ab = (size_t)6 * ch.nh * real_bytes(c->prec);
  CK(cudaMemcpyAsync(ch.uf, ch.u, ub, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(ch.af, ch.a, ab, cudaMemcpyDeviceToDevice, c->stream));
  return gf_loop(c, chain, theta, iters, max_iters);
}

int lce_gauge_fix_continue(lce_ctx* c, int chain, double* theta, int* iters, int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  return gf_loop(c, chain, theta, iters, max_iters);
}

int lce_it_gauge_fixing(lce_ctx* c, int chain, double step, int flags, double* da1) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains || (flags & ~(LCE_ITGF_FIX_COMPONENT | LCE_ITGF_ASCEND | LCE_ITGF_TRACK)))
    return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  ChainState cs;
  CK(cudaMemcpyAsync(&cs, c->cst_d + chain, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  cs.gf_done = 0;
  cs.gf_iters = 0;
  cs.gf_cap = 1;
  cs.gf_theta = 1.0e4;
  cs.gf_step = step > 0.0 ? step : ch.alpha;
  CK(cudaMemcpyAsync(c->cst_d + chain, &cs, sizeof(cs), cudaMemcpyHostToDevice, c->stream));
  // the subroutine itself: no reunitarisation
  if (c->prec == LCE_PREC_F64)
    launch_it_iteration<double>(c->ch_d + chain, c->cst_d + chain, flags, 0, c->scratch_d, ch.nh, c->stream);
  else
    launch_it_iteration<float>(c->ch_d + chain, c->cst_d + chain, flags, 0, c->scratch_d, ch.nh, c->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&cs, c->cst_d + chain, sizeof(cs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (da1) *da1 = cs.gf_theta;
  if (!std::isfinite(cs.gf_theta)) return fail(c, LCE_ERR_NAN, "it_gauge_fixing: da1 is not finite");
  return LCE_OK;
}

int lce_it_landau_gauge(lce_ctx* c, int chain, double step, int flags, double* da1, int* iters, int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains || (flags & ~(LCE_ITGF_FIX_COMPONENT | LCE_ITGF_ASCEND | LCE_ITGF_TRACK)))
    return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  const size_t ub = (size_t)6 * ch.nh * link_bytes(c->prec), ab = (size_t)6 * ch.nh * real_bytes(c->prec);
  CK(cudaMemcpyAsync(ch.uf, ch.u, ub, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(ch.af, ch.a, ab, cudaMemcpyDeviceToDevice, c->stream));
  if (flags & LCE_ITGF_TRACK) {
    if (c->prec == LCE_PREC_F64) launch_transform_identity<double>(ch.g, ch.nh, c->stream);
    else launch_transform_identity<float>(ch.g, ch.nh, c->stream);
  }
  return gf_loop(c, chain, da1, iters, max_iters, 0, flags, step > 0.0 ? step : ch.alpha);
}

int lce_apply_transform(lce_ctx* c, int chain) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  if (c->prec == LCE_PREC_F64) launch_gauge_apply<double>(c->ch_d + chain, c->ch[chain].nh, c->stream);
  else launch_gauge_apply<float>(c->ch_d + chain, c->ch[chain].nh, c->stream);
  CK(cudaGetLastError());
  return LCE_OK;
}

int lce_landau_gauge_from(lce_ctx* c, int chain, int start, double* theta_start, double* theta, int* iters,
                          int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  if (start == LCE_GF_START_IDENTITY) {
    if (c->prec == LCE_PREC_F64) launch_transform_identity<double>(ch.g, ch.nh, c->stream);
    else launch_transform_identity<float>(ch.g, ch.nh, c->stream);
    const size_t ub = (size_t)6 * ch.nh * link_bytes(c->prec), ab = (size_t)6 * ch.nh * real_bytes(c->prec);
    CK(cudaMemcpyAsync(ch.uf, ch.u, ub, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(ch.af, ch.a, ab, cudaMemcpyDeviceToDevice, c->stream));
  } else if (start == LCE_GF_START_TRANSFORM) {
    int rc = lce_apply_transform(c, chain);
    if (rc) return rc;
  } else {
    return fail(c, LCE_ERR_INVALID, "landau_gauge_from: unknown start");
  }
  if (theta_start) {
    int rc = lce_theta(c, chain, theta_start);
    if (rc) return rc;
  }
  return gf_loop(c, chain, theta, iters, max_iters, 1);
}

int lce_landau_gauge_warm(lce_ctx* c, int chain, lce_net* net, int flags, int* start_used, double functional[3],
                          double* theta, int* iters, int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains ||
      (flags & ~(LCE_WARM_NET | LCE_WARM_JUDGE | LCE_WARM_RECORD | LCE_WARM_FOURIER | LCE_WARM_CG)))
    return LCE_ERR_INVALID;
  const bool use_net = flags & LCE_WARM_NET, judge = flags & LCE_WARM_JUDGE, record = flags & LCE_WARM_RECORD;
  if ((use_net || record) && !net) return fail(c, LCE_ERR_INVALID, "landau_gauge_warm: no network given");
  if (net && net_device(net) != c->device) return fail(c, LCE_ERR_INVALID, "landau_gauge_warm: network on another device");
  const ChainDev& ch = c->ch[chain];
  const bool f64 = c->prec == LCE_PREC_F64;
  const bool fourier = flags & LCE_WARM_FOURIER;
  if (fourier && !fa_supported(ch))
    return fail(c, LCE_ERR_UNSUPPORTED, "Fourier-accelerated fixing needs power-of-two extents");
  const size_t gb = (size_t)2 * ch.nh * link_bytes(c->prec);
  if (!c->gsave_d) CK(cudaMalloc(&c->gsave_d, (size_t)2 * c->max_nh * link_bytes(c->prec)));
  double F[3] = {NAN, NAN, NAN};
  int rc;
  // candidate 1: G_prev
  CK(cudaMemcpyAsync(c->gsave_d, ch.g, gb, cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = lce_apply_transform(c, chain))) return rc;
  if (judge && (rc = lce_gauge_functional(c, chain, &F[1]))) return rc;
  if (use_net || record) {
    if ((rc = net_features(net, c->ch_d + chain, ch, f64, c->stream))) return fail(c, rc, "network features");
  }
  // candidate 2: Omega G_prev
  if (use_net) {
    net_predict(net, ch, c->stream);
    if (judge) {
      if ((rc = net_compose(net, ch, c->gsave_d, f64, c->stream))) return fail(c, rc, "network compose");
      if ((rc = lce_apply_transform(c, chain))) return rc;
      if ((rc = lce_gauge_functional(c, chain, &F[2]))) return rc;
    }
  }
  // candidate 0: the identity, the reference's start
  if (judge) {
    const size_t ub = (size_t)6 * ch.nh * link_bytes(c->prec), ab = (size_t)6 * ch.nh * real_bytes(c->prec);
    CK(cudaMemcpyAsync(ch.uf, ch.u, ub, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(ch.af, ch.a, ab, cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = lce_gauge_functional(c, chain, &F[0]))) return rc;
  }
  int pick = use_net ? LCE_GF_START_NET : LCE_GF_START_TRANSFORM;
  if (judge) {
    pick = LCE_GF_START_IDENTITY;
    if (F[1] > F[pick]) pick = LCE_GF_START_TRANSFORM;
    if (use_net && F[2] > F[pick]) pick = LCE_GF_START_NET;
  }
  if (pick == LCE_GF_START_IDENTITY) {
    // U_f, A_f already hold U, A
    if (f64) launch_transform_identity<double>(ch.g, ch.nh, c->stream);
    else launch_transform_identity<float>(ch.g, ch.nh, c->stream);
  } else {
    if (pick == LCE_GF_START_TRANSFORM) {
      CK(cudaMemcpyAsync(ch.g, c->gsave_d, gb, cudaMemcpyDeviceToDevice, c->stream));
    } else if ((rc = net_compose(net, ch, c->gsave_d, f64, c->stream))) {
      return fail(c, rc, "network compose");
    }
    if ((rc = lce_apply_transform(c, chain))) return rc;
  }
  CK(cudaGetLastError());
  if (start_used) *start_used = pick;
  if (functional)
    for (int k = 0; k < 3; ++k) functional[k] = F[k];
  if (fourier) {
    const int cap = max_iters > 0 ? max_iters : 1000000;
    double th = 0.0;
    int it = 0;
    rc = fa_loop(c, chain, 1.0, ch.limit_or, &th, &it, cap, (flags & LCE_WARM_CG) != 0);
    if (theta) *theta = th;
    if (iters) *iters = it;
    if (rc == LCE_OK && th > ch.limit_or) rc = fail(c, LCE_ERR_GF_NOT_CONVERGED, "gauge fixing: iteration cap reached");
  } else {
    rc = gf_loop(c, chain, theta, iters, max_iters, 1);
  }
  if (rc == LCE_OK && record) {
    if ((rc = net_record(net, ch, c->gsave_d, f64, c->stream))) return fail(c, rc, "record training pair");
    CK(cudaStreamSynchronize(c->stream));
  }
  if (rc == LCE_OK && use_net) {
    CK(cudaStreamSynchronize(c->stream));
    if ((rc = net_status(net))) return fail(c, rc, lce_last_error(nullptr));
  }
  return rc;
}

}  // extern "C"

namespace {
int fourier_fix(lce_ctx* c, int chain, int start, double step, double theta_switch, double* theta,
                int* iters_fourier, int* iters_plain, int max_iters, bool cg) {
  const ChainDev& ch = c->ch[chain];
  if (!fa_supported(ch)) return fail(c, LCE_ERR_UNSUPPORTED, "Fourier-accelerated fixing needs power-of-two extents");
  if (!(step > 0.0)) step = 1.0;
  if (!(theta_switch > 0.0)) theta_switch = ch.limit_or;
  if (start == LCE_GF_START_IDENTITY) {
    if (c->prec == LCE_PREC_F64) launch_transform_identity<double>(ch.g, ch.nh, c->stream);
    else launch_transform_identity<float>(ch.g, ch.nh, c->stream);
    const size_t ub = (size_t)6 * ch.nh * link_bytes(c->prec), ab = (size_t)6 * ch.nh * real_bytes(c->prec);
    CK(cudaMemcpyAsync(ch.uf, ch.u, ub, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(ch.af, ch.a, ab, cudaMemcpyDeviceToDevice, c->stream));
  } else if (start == LCE_GF_START_TRANSFORM) {
    int rc = lce_apply_transform(c, chain);
    if (rc) return rc;
  } else {
    return fail(c, LCE_ERR_INVALID, "landau_gauge_fourier: unknown start");
  }
  const int cap = max_iters > 0 ? max_iters : 1000000;
  double th_fa = 0.0;
  int it_fa = 0, it_or = 0;
  int rc = fa_loop(c, chain, step, theta_switch, &th_fa, &it_fa, cap, cg);
  if (iters_fourier) *iters_fourier = it_fa;
  if (iters_plain) *iters_plain = 0;
  if (theta) *theta = th_fa;
  if (rc) return rc;
  if (th_fa <= ch.limit_or) return LCE_OK;
  if (it_fa >= cap) return fail(c, LCE_ERR_GF_NOT_CONVERGED, "Fourier-accelerated fixing: iteration cap reached");
  // the plain overrelaxed iteration from theta_switch to limit_or
  rc = gf_loop(c, chain, theta, &it_or, cap - it_fa, 1);
  if (iters_plain) *iters_plain = it_or;
  return rc;
}
}  // namespace

extern "C" {

int lce_landau_gauge_fourier(lce_ctx* c, int chain, int start, double step, double theta_switch, double* theta,
                             int* iters_fourier, int* iters_plain, int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  return fourier_fix(c, chain, start, step, theta_switch, theta, iters_fourier, iters_plain, max_iters, false);
}

int lce_landau_gauge_fourier_cg(lce_ctx* c, int chain, int start, double theta_switch, double* theta,
                                int* iters_fourier, int* iters_plain, int max_iters) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  return fourier_fix(c, chain, start, 1.0, theta_switch, theta, iters_fourier, iters_plain, max_iters, true);
}

int lce_debug_fourier_step(lce_ctx* c, int chain, double step, double* omega) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !omega || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  if (!fa_supported(ch)) return fail(c, LCE_ERR_UNSUPPORTED, "power-of-two extents needed");
  int rc = fa_buffers(c);
  if (rc) return rc;
  double* om = nullptr;
  const size_t ob = sizeof(double) * 3 * 2 * (size_t)ch.nh;
  CK(cudaMalloc(&om, ob));
  if (c->prec == LCE_PREC_F64)
    launch_fa_iteration<double>(c->ch_d + chain, ch, nullptr, step, c->fa_d, fa_vcap(c), c->scratch_d, om, 0, false,
                                false, false, c->stream);
  else
    launch_fa_iteration<float>(c->ch_d + chain, ch, nullptr, step, c->fa_d, fa_vcap(c), c->scratch_d, om, 0, false,
                               false, false, c->stream);
  cudaError_t e = cudaGetLastError();
  const std::string fe = fa_take_error();
  if (e == cudaSuccess && fe.empty()) e = cudaMemcpyAsync(omega, om, ob, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && fe.empty()) e = cudaStreamSynchronize(c->stream);
  cudaFree(om);
  if (!fe.empty()) return fail(c, LCE_ERR_CUDA, "debug_fourier_step: " + fe);
  if (e != cudaSuccess) return cuda_fail(c, e, "debug_fourier_step");
  return LCE_OK;
}

int lce_set_transform(lce_ctx* c, int chain, const float* g, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !g || chain < 0 || chain >= c->nchains || ld < c->ch[chain].nh) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  const int nh = ch.nh;
  if (c->prec == LCE_PREC_F32) {
    CK(cudaMemcpy2DAsync(ch.g, (size_t)nh * 16, g, (size_t)ld * 16, (size_t)nh * 16, 2, cudaMemcpyHostToDevice,
                         c->stream));
  } else {
    std::vector<double> h((size_t)2 * nh * 4);
    for (int eo = 0; eo < 2; ++eo)
      for (long i = 0; i < (long)nh * 4; ++i) h[(size_t)eo * nh * 4 + i] = g[(size_t)eo * ld * 4 + i];
    CK(cudaMemcpyAsync(ch.g, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return LCE_OK;
}

int lce_get_transform(lce_ctx* c, int chain, float* g, long ld) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !g || chain < 0 || chain >= c->nchains || ld < c->ch[chain].nh) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  const int nh = ch.nh;
  if (c->prec == LCE_PREC_F32) {
    CK(cudaMemcpy2DAsync(g, (size_t)ld * 16, ch.g, (size_t)nh * 16, (size_t)nh * 16, 2, cudaMemcpyDeviceToHost,
                         c->stream));
    CK(cudaStreamSynchronize(c->stream));
  } else {
    std::vector<double> h((size_t)2 * nh * 4);
    CK(cudaMemcpyAsync(h.data(), ch.g, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int eo = 0; eo < 2; ++eo)
      for (long i = 0; i < (long)nh * 4; ++i) g[(size_t)eo * ld * 4 + i] = (float)h[(size_t)eo * nh * 4 + i];
  }
  return LCE_OK;
}

int lce_gauge_functional(lce_ctx* c, int chain, double* value) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !value || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  const int nb = ceil_div(2L * ch.nh, 256);
  double* part = c->scratch_d;
  double* out = c->scratch_d + nb;
  if (c->prec == LCE_PREC_F64) launch_functional<double>(c->ch_d + chain, part, ch.nh, c->stream);
  else launch_functional<float>(c->ch_d + chain, part, ch.nh, c->stream);
  launch_sum_partials(part, nb, 1, out, c->stream);
  CK(cudaGetLastError());
  double s;
  CK(cudaMemcpyAsync(&s, out, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *value = s / ((2.0 + ch.alpha) * 2.0 * ch.nh);
  return LCE_OK;
}

int lce_theta(lce_ctx* c, int chain, double* theta) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !theta || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  const int nb = ceil_div(ch.nh, kBlock);
  double* part = c->scratch_d;
  double* out = c->scratch_d + nb;
  if (c->prec == LCE_PREC_F64) launch_gf_theta<double>(c->ch_d + chain, part, ch.nh, c->stream);
  else launch_gf_theta<float>(c->ch_d + chain, part, ch.nh, c->stream);
  launch_sum_partials(part, nb, 1, out, c->stream);
  CK(cudaGetLastError());
  double s;
  CK(cudaMemcpyAsync(&s, out, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *theta = s / ch.nh;
  return LCE_OK;
}

int lce_correlator(lce_ctx* c, int chain, double* corr_a, double* corr_u, double* corr_3, double af[3]) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const int L3 = c->ch[chain].L3;
  double* out;
  int rc = get_slices(c, chain, out);
  if (rc) return rc;
  std::vector<double> h((size_t)7 * L3 + 5);
  CK(cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (corr_a) std::memcpy(corr_a, h.data(), L3 * sizeof(double));
  if (corr_u) std::memcpy(corr_u, h.data() + L3, L3 * sizeof(double));
  if (corr_3) std::memcpy(corr_3, h.data() + 2 * L3, L3 * sizeof(double));
  if (af) std::memcpy(af, h.data() + 7 * L3, 3 * sizeof(double));
  return LCE_OK;
}

int lce_polyakov(lce_ctx* c, int chain, double* slice, double* corr, double* mean2) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const int L3 = c->ch[chain].L3;
  double* out;
  int rc = get_slices(c, chain, out);
  if (rc) return rc;
  std::vector<double> h((size_t)7 * L3 + 5);
  CK(cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (slice) std::memcpy(slice, h.data() + 3 * L3, L3 * sizeof(double));
  if (corr) std::memcpy(corr, h.data() + 4 * L3, L3 * sizeof(double));
  if (mean2) *mean2 = h[7 * L3 + 3];
  return LCE_OK;
}

int lce_scalarcorr(lce_ctx* c, int chain, double* slice, double* corr, double* mean) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const int L3 = c->ch[chain].L3;
  double* out;
  int rc = get_slices(c, chain, out);
  if (rc) return rc;
  std::vector<double> h((size_t)7 * L3 + 5);
  CK(cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (slice) std::memcpy(slice, h.data() + 5 * L3, L3 * sizeof(double));
  if (corr) std::memcpy(corr, h.data() + 6 * L3, L3 * sizeof(double));
  if (mean) *mean = h[7 * L3 + 4];
  return LCE_OK;
}

int lce_plaquette(lce_ctx* c, int chain, double* plaq) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !plaq || chain < 0 || chain >= c->nchains) return LCE_ERR_INVALID;
  const ChainDev& ch = c->ch[chain];
  const int nb = ceil_div(2L * ch.nh, 256);
  double* part = c->scratch_d;
  double* out = c->scratch_d + nb;
  if (c->prec == LCE_PREC_F64) launch_plaquette<double>(c->ch_d + chain, part, ch.nh, c->stream);
  else launch_plaquette<float>(c->ch_d + chain, part, ch.nh, c->stream);
  launch_sum_partials(part, nb, 1, out, c->stream);
  CK(cudaGetLastError());
  double s;
  CK(cudaMemcpyAsync(&s, out, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *plaq = s / (3.0 * 2.0 * ch.nh);
  return LCE_OK;
}

int lce_debug_staple(lce_ctx* c, int eo, int mu, double* out) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !out || eo < 0 || eo > 1 || mu < 0 || mu > 2) return LCE_ERR_INVALID;
  const int nh = c->ch[0].nh;
  int rc = ensure_staging(c, (size_t)nh * 4 * sizeof(double));
  if (rc) return rc;
  if (c->prec == LCE_PREC_F64) launch_debug_staple<double>(c->ch_d, eo, mu, (double*)c->staging_d, nh, c->stream);
  else launch_debug_staple<float>(c->ch_d, eo, mu, (double*)c->staging_d, nh, c->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->staging_d, (size_t)nh * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return LCE_OK;
}

int lce_debug_force(lce_ctx* c, int eo, double* out) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !out || eo < 0 || eo > 1) return LCE_ERR_INVALID;
  const int nh = c->ch[0].nh;
  int rc = ensure_staging(c, (size_t)nh * 3 * sizeof(double));
  if (rc) return rc;
  if (c->prec == LCE_PREC_F64) launch_debug_force<double>(c->ch_d, eo, (double*)c->staging_d, nh, c->stream);
  else launch_debug_force<float>(c->ch_d, eo, (double*)c->staging_d, nh, c->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->staging_d, (size_t)nh * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return LCE_OK;
}

int lce_flush_l2(lce_ctx* c) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  if (!c->flush_d) {
    c->flush_bytes = (size_t)256 << 20;  // written; a second 256 MB half is read
    CK(cudaMalloc(&c->flush_d, 2 * c->flush_bytes));
  }
  launch_flush(c->flush_d, c->flush_bytes, c->stream);
  CK(cudaGetLastError());
  return LCE_OK;
}

// One sweep of the per-pass form as a CUDA graph whose pass kernels are timed
// without being disturbed: after pass i an event-record node on a side stream
// fires when the pass has completed, while pass i + 1 keeps its
// programmatic-dependent-launch edge to pass i (the timing nodes hang off the
// kernel chain instead of sitting on it, as events between the launches
// would).  ms[i] = completion of pass i minus completion of pass i - 1 (pass
// 0: from the graph's start), ms[npasses] = the finalize kernel's; returns
// the pass count.  The graph is built once per measflag and tile shape.
int lce_profile_sweep(lce_ctx* c, int measflag, float* ms, int max_passes) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !ms || max_passes < 1) return LCE_ERR_INVALID;
  const int mf = measflag == 1 ? 1 : 0;
  const std::vector<unsigned char> r = sweep_routines(c);
  std::vector<Pass> passes;
  for (unsigned char k : r) expand(k, passes);
  const int np = (int)passes.size();
  if (!c->side) {
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming));
  }
  while ((int)c->prof_ev.size() < np + 2) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    c->prof_ev.push_back(e);
  }
  cudaGraphExec_t* slot = &c->sweep_graphs[std::make_tuple(-1, c->tile_bs, c->tile_spt, c->tile_occ, mf, 1)];
  if (!*slot) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaEventRecordWithFlags(c->prof_ev[0], c->stream, cudaEventRecordExternal);
    Enq q;
    int rc = LCE_OK;
    if (e == cudaSuccess) {
      enq_begin(c, r, mf, true, c->tile_bs, c->tile_spt, c->tile_occ, q);
      for (int i = 0; i < np && rc == LCE_OK && e == cudaSuccess; ++i) {
        rc = enq_pass(c, q, i);
        if (rc == LCE_OK) e = cudaEventRecord(c->fork_ev, c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->side, c->fork_ev, 0);
        if (e == cudaSuccess) e = cudaEventRecordWithFlags(c->prof_ev[i + 1], c->side, cudaEventRecordExternal);
      }
      if (rc == LCE_OK && e == cudaSuccess) rc = enq_end(c, q);
      if (rc == LCE_OK && e == cudaSuccess)
        e = cudaEventRecordWithFlags(c->prof_ev[np + 1], c->stream, cudaEventRecordExternal);
    }
    // rejoin the side stream whatever happened, so that the capture can end
    const cudaError_t ej1 = cudaEventRecord(c->join_ev, c->side);
    const cudaError_t ej2 = cudaStreamWaitEvent(c->stream, c->join_ev, 0);
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    cudaError_t ei = cudaSuccess;
    if (ec == cudaSuccess) {
      if (rc == LCE_OK && e == cudaSuccess && ej1 == cudaSuccess && ej2 == cudaSuccess)
        ei = cudaGraphInstantiate(slot, g, 0);
      cudaGraphDestroy(g);
    }
    if (rc) return rc;
    for (cudaError_t x : {e, ej1, ej2, ec, ei})
      if (x != cudaSuccess) {
        *slot = nullptr;
        cudaGetLastError();
        return cuda_fail(c, x, "profile_sweep graph");
      }
  }
  CK(cudaGraphLaunch(*slot, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i <= np && i < max_passes; ++i) CK(cudaEventElapsedTime(&ms[i], c->prof_ev[i], c->prof_ev[i + 1]));
  return np;
}

int lce_timer_start(lce_ctx* c) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c) return LCE_ERR_INVALID;
  CK(cudaEventRecord(c->ev0, c->stream));
  return LCE_OK;
}

int lce_timer_stop(lce_ctx* c, float* ms) {
  DeviceScope ds_(c ? c->device : -1);
  if (!c || !ms) return LCE_ERR_INVALID;
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return LCE_OK;
}

// ---- z-slab decomposition
lce_slabs* lce_slabs_create(const lce_params* p, int nslabs, const int* devices) {
  g_create_error.clear();
  if (!p || nslabs < 1 || !devices) {
    slabs_fail(LCE_ERR_INVALID, "slabs_create: null params or devices, or no slabs");
    return nullptr;
  }
  std::string why;
  if (!valid_params(*p, why)) {
    slabs_fail(LCE_ERR_INVALID, "slabs_create: " + why);
    return nullptr;
  }
  const int L3 = p->L[2], nz = L3 / nslabs;
  if (L3 % nslabs != 0 || nz < 2 || (nz & 1)) {
    slabs_fail(LCE_ERR_INVALID, "slabs_create: L3 must split into slabs of an even number (>= 2) of planes");
    return nullptr;
  }
  if (p->rng == LCE_RNG_STREAM && p->precision != LCE_PREC_F64) {
    slabs_fail(LCE_ERR_UNSUPPORTED, "slabs_create: validation streams need LCE_PREC_F64");
    return nullptr;
  }
  if ((size_t)L3 * 14 * sizeof(double) > 200 * 1024) {
    slabs_fail(LCE_ERR_INVALID, "slabs_create: L3 too large for the correlator kernel");
    return nullptr;
  }
  lce_slabs* S = new lce_slabs();
  S->L[0] = p->L[0];
  S->L[1] = p->L[1];
  S->L[2] = L3;
  S->nz = nz;
  S->nxy = p->L[0] * p->L[1] / 2;
  S->prec = p->precision;
  S->delta = p->delta0;
  for (int k = 0; k < nslabs; ++k) {
    lce_params q = *p;
    q.L[2] = nz + 2;
    q.device = devices[k];
    q.sweep_mode = LCE_SWEEP_PASSES;
    const int z0 = k * nz;
    const SlabInfo si{(z0 - 1) * S->nxy, (z0 + 1) & 1, S->nxy * L3};
    DeviceScope ds_(devices[k]);
    lce_ctx* c = create_impl(&q, 1, &si);
    if (!c) {
      const std::string m = "slabs_create: slab " + std::to_string(k) + ": " + g_create_error;
      lce_slabs_destroy(S);
      slabs_fail(LCE_ERR_CUDA, m);
      g_create_error = m;
      return nullptr;
    }
    S->slab.push_back(c);
    cudaEvent_t e1 = nullptr, e2 = nullptr;
    if (cudaEventCreateWithFlags(&e1, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e2, cudaEventDisableTiming) != cudaSuccess) {
      if (e1) cudaEventDestroy(e1);
      lce_slabs_destroy(S);
      g_create_error = "slabs_create: cudaEventCreate";
      slabs_fail(LCE_ERR_CUDA, g_create_error);
      return nullptr;
    }
    S->ev_pass.push_back(e1);
    S->ev_copy.push_back(e2);
    cudaEvent_t e3 = nullptr;
    if (cudaEventCreateWithFlags(&e3, cudaEventDisableTiming) != cudaSuccess) {
      lce_slabs_destroy(S);
      g_create_error = "slabs_create: cudaEventCreate";
      slabs_fail(LCE_ERR_CUDA, g_create_error);
      return nullptr;
    }
    S->ev_sum.push_back(e3);
  }
  {
    // theta sums, slice sums and correlators of the whole lattice on slab 0's device
    DeviceScope ds_(devices[0]);
    const size_t gn = (size_t)nslabs + (size_t)21 * L3 + 5;
    if (cudaEventCreateWithFlags(&S->ev_chk, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&S->g_d, gn * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      S->g_d = nullptr;
      lce_slabs_destroy(S);
      g_create_error = "slabs_create: slab 0 gather buffer";
      slabs_fail(LCE_ERR_NOMEM, g_create_error);
      return nullptr;
    }
  }
  // direct peer copies between the devices that hold neighbouring slabs
  for (int k = 0; k < nslabs; ++k) {
    const int d0 = devices[k], d1 = devices[(k + 1) % nslabs];
    if (d0 == d1) continue;
    int ok01 = 0, ok10 = 0;
    cudaDeviceCanAccessPeer(&ok01, d0, d1);
    cudaDeviceCanAccessPeer(&ok10, d1, d0);
    if (ok01) {
      DeviceScope ds_(d0);
      if (cudaDeviceEnablePeerAccess(d1, 0) != cudaSuccess) cudaGetLastError();  // already enabled is fine
    }
    if (ok10) {
      DeviceScope ds_(d1);
      if (cudaDeviceEnablePeerAccess(d0, 0) != cudaSuccess) cudaGetLastError();
    }
  }
  return S;
}

void lce_slabs_destroy(lce_slabs* h) {
  lce_slabs* S = h;
  if (!S) return;
  if (!S->slab.empty()) {
    DeviceScope ds_(S->slab[0]->device);
    if (S->g_d) cudaFree(S->g_d);
    if (S->fft_d) cudaFree(S->fft_d);
    if (S->cg_d) cudaFree(S->cg_d);
    if (S->ev_chk) cudaEventDestroy(S->ev_chk);
  }
  for (size_t k = 0; k < S->slab.size(); ++k) {
    DeviceScope ds_(S->slab[k]->device);
    if (k < S->ev_pass.size()) cudaEventDestroy(S->ev_pass[k]);
    if (k < S->ev_copy.size()) cudaEventDestroy(S->ev_copy[k]);
    if (k < S->ev_sum.size()) cudaEventDestroy(S->ev_sum[k]);
    lce_destroy(S->slab[k]);
  }
  delete S;
}

int lce_slabs_upload(lce_slabs* h, const float* u, const float* a, long ld) {
  lce_slabs* S = h;
  if (!S || !u || !a || ld < (long)S->nxy * S->L[2]) return LCE_ERR_INVALID;
  return slabs_copy<float>(S, const_cast<float*>(u), const_cast<float*>(a), ld, true);
}

int lce_slabs_upload_f64(lce_slabs* h, const double* u, const double* a, long ld) {
  lce_slabs* S = h;
  if (!S || !u || !a || ld < (long)S->nxy * S->L[2]) return LCE_ERR_INVALID;
  return slabs_copy<double>(S, const_cast<double*>(u), const_cast<double*>(a), ld, true);
}

int lce_slabs_download(lce_slabs* h, float* u, float* a, long ld) {
  lce_slabs* S = h;
  if (!S || !u || !a || ld < (long)S->nxy * S->L[2]) return LCE_ERR_INVALID;
  return slabs_copy<float>(S, u, a, ld, false);
}

int lce_slabs_download_f64(lce_slabs* h, double* u, double* a, long ld) {
  lce_slabs* S = h;
  if (!S || !u || !a || ld < (long)S->nxy * S->L[2]) return LCE_ERR_INVALID;
  return slabs_copy<double>(S, u, a, ld, false);
}

int lce_slabs_set_rng_stream(lce_slabs* h, const double* u, size_t n) {
  if (!h || (!u && n)) return slabs_fail(LCE_ERR_INVALID, "slabs_set_rng_stream: null stream");
  for (lce_ctx* c : h->slab) {
    DeviceScope ds_(c->device);
    if (int rc = lce_set_rng_stream(c, u, n)) return slab_rc(c, rc);
  }
  return LCE_OK;
}

int lce_slabs_sweep(lce_slabs* h, int measflag, lce_meas* m) {
  lce_slabs* S = h;
  if (!S || (measflag != 0 && measflag != 1)) return LCE_ERR_INVALID;
  return slab_sweep(S, measflag, m);
}

int lce_slabs_download_fixed(lce_slabs* h, float* u, float* a, long ld) {
  lce_slabs* S = h;
  if (!S || !u || !a || ld < (long)S->nxy * S->L[2]) return LCE_ERR_INVALID;
  return slabs_copy<float>(S, u, a, ld, false, LCE_FIELDS_FIXED);
}

int lce_slabs_download_fixed_f64(lce_slabs* h, double* u, double* a, long ld) {
  lce_slabs* S = h;
  if (!S || !u || !a || ld < (long)S->nxy * S->L[2]) return LCE_ERR_INVALID;
  return slabs_copy<double>(S, u, a, ld, false, LCE_FIELDS_FIXED);
}

int lce_slabs_landau_gauge(lce_slabs* h, double* theta, int* iters, int max_iters) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  return slab_landau_gauge(S, theta, iters, max_iters);
}

int lce_slabs_it_landau_gauge(lce_slabs* h, double step, int flags, double* da1, int* iters, int max_iters) {
  lce_slabs* S = h;
  if (!S || (flags & ~(LCE_ITGF_FIX_COMPONENT | LCE_ITGF_ASCEND | LCE_ITGF_TRACK))) return LCE_ERR_INVALID;
  lce_ctx* c0 = S->slab[0];
  const int cap = max_iters > 0 ? max_iters : 1000000;
  if (int rc = slab_gf_start(S, (flags & LCE_ITGF_TRACK) ? LCE_GF_START_IDENTITY : -1)) return rc;
  if (int rc = slab_gf_state(S, cap, -1.0, step > 0.0 ? step : c0->ch[0].alpha)) return rc;
  ChainState cs;
  if (int rc = slab_gf_run(S, 0, false, cs, flags)) return rc;
  if (da1) *da1 = cs.gf_theta;
  if (iters) *iters = cs.gf_iters;
  if (!std::isfinite(cs.gf_theta)) return slabs_fail(LCE_ERR_NAN, "slabs gauge fixing: da1 is not finite");
  if (cs.gf_theta > c0->ch[0].limit_or)
    return slabs_fail(LCE_ERR_GF_NOT_CONVERGED, "slabs gauge fixing: iteration cap reached");
  return LCE_OK;
}

int lce_slabs_landau_gauge_fourier(lce_slabs* h, int start, double step, double theta_switch, double* theta,
                                   int* iters_fourier, int* iters_plain, int max_iters) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  if (start != LCE_GF_START_IDENTITY && start != LCE_GF_START_TRANSFORM)
    return slabs_fail(LCE_ERR_INVALID, "slabs_landau_gauge_fourier: start must be IDENTITY or TRANSFORM");
  return slab_fourier_fix(S, start, step, theta_switch, theta, iters_fourier, iters_plain, max_iters);
}

int lce_slabs_landau_gauge_fourier_cg(lce_slabs* h, int start, double theta_switch, double* theta,
                                      int* iters_fourier, int* iters_plain, int max_iters) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  if (start != LCE_GF_START_IDENTITY && start != LCE_GF_START_TRANSFORM)
    return slabs_fail(LCE_ERR_INVALID, "slabs_landau_gauge_fourier_cg: start must be IDENTITY or TRANSFORM");
  return slab_fourier_fix(S, start, 1.0, theta_switch, theta, iters_fourier, iters_plain, max_iters, true);
}

int lce_slabs_landau_gauge_from(lce_slabs* h, int start, double* theta, int* iters, int max_iters) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  if (start != LCE_GF_START_IDENTITY && start != LCE_GF_START_TRANSFORM)
    return slabs_fail(LCE_ERR_INVALID, "slabs_landau_gauge_from: start must be IDENTITY or TRANSFORM");
  return slab_landau_gauge(S, theta, iters, max_iters, start);
}

int lce_slabs_correlator(lce_slabs* h, double* corr_a, double* corr_u, double* corr_3, double af[3]) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  std::vector<double> v;
  if (int rc = slab_slices(S, v)) return rc;
  const int L3 = S->L[2];
  if (corr_a) std::memcpy(corr_a, v.data(), L3 * sizeof(double));
  if (corr_u) std::memcpy(corr_u, v.data() + L3, L3 * sizeof(double));
  if (corr_3) std::memcpy(corr_3, v.data() + 2 * L3, L3 * sizeof(double));
  if (af) std::memcpy(af, v.data() + 7 * L3, 3 * sizeof(double));
  return LCE_OK;
}

int lce_slabs_polyakov(lce_slabs* h, double* slice, double* corr, double* mean2) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  std::vector<double> v;
  if (int rc = slab_slices(S, v)) return rc;
  const int L3 = S->L[2];
  if (slice) std::memcpy(slice, v.data() + 3 * L3, L3 * sizeof(double));
  if (corr) std::memcpy(corr, v.data() + 4 * L3, L3 * sizeof(double));
  if (mean2) *mean2 = v[7 * L3 + 3];
  return LCE_OK;
}

int lce_slabs_scalarcorr(lce_slabs* h, double* slice, double* corr, double* mean) {
  lce_slabs* S = h;
  if (!S) return LCE_ERR_INVALID;
  std::vector<double> v;
  if (int rc = slab_slices(S, v)) return rc;
  const int L3 = S->L[2];
  if (slice) std::memcpy(slice, v.data() + 5 * L3, L3 * sizeof(double));
  if (corr) std::memcpy(corr, v.data() + 6 * L3, L3 * sizeof(double));
  if (mean) *mean = v[7 * L3 + 4];
  return LCE_OK;
}

}  // extern "C"
