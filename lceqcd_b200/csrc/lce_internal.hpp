// lce_internal.hpp -- descriptors shared by the kernels and the C-ABI layer.
//
// Device layout of one chain (all planes 256-byte aligned, one allocation):
//   U   [mu 0..2][parity 0..1][site 0..nh-1]  links, float4 or 2 x double2
//   A   [parity][k 0..2][site]                adjoint Higgs, SoA planes
//   U_f, A_f                                  gauge-fixed copies, same layout
// "parity" is the reference's eo index; sites inside a parity are in the
// half-row order of f/adresses.f.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "lce_common.cuh"
#include "../../include/lceqcd_gpu.h"

namespace lce {

constexpr int kBlock = 256;      // threads per block of the update kernels
// resident blocks per SM the update kernels are compiled for (register cap
// 64 for FP32 production kernels, 80 for the FP64 validation kernels).  FP32:
// 4 blocks of 256 (64 registers) keep a 64^3 parity pass (131,072 sites) in one
// wave on 148 SMs and let the compiler issue the staple loads together; timed
// on a B200 it beats 5 (48 registers, spills), 3 (80) and 2 (92) blocks at
// every volume from 64^3 to 256^3 (by 17% at 64^3, 3-6% at 128^3-256^3).
template <typename R>
constexpr int min_blocks() { return sizeof(R) == 4 ? 4 : 3; }
constexpr int kNQ = 4;           // doubles of partial sums per block
constexpr int kMaxSlots = 64;    // reduction slots per finalize
constexpr int kChunkTiles = 128; // tiles per level-1 chunk of the finalize reduction
// the tile sizes (sites) of the per-pass kernels' tile tables: 448 = 14 warps,
// two blocks per SM, balances a single-wave pass (a 64^3 parity: 293 blocks
// on 148 SMs, at most 28 warps on an SM against 32 with 512)
constexpr int kTileTables = 4;  // (CtxState::rb_chunk_begin has one entry per table)
constexpr int kTileSites[kTileTables] = {128, 256, 512, 448};

// pass kinds (one kernel launch over one parity)
enum PassKind : unsigned char {
  kHiggsHB = 0,     // ahiggs2
  kHiggsOR = 1,     // ahiggs3
  kHiggsMetro = 2,  // ahiggs1
  kLinkHB = 3,      // agauge
  kLinkOR = 4,      // link overrelaxation (no reference counterpart)
  kLinkHB3 = 5,     // agauge of f/agauge1.f: three heatbath + Metropolis hits
  kKindEnd = 0x80,  // flag: last slot of one routine
};

struct ChainDev {
  int L1, L2, L3, hx, nxy, nh;
  FastDiv dhx, dnxy;
  double beta, beta_a, beta_2, beta_4, lambda, alpha, limit_or;
  double inv_beta2, cxval0;  // 1/beta_2 and 1/beta_2/2 in the fields' precision
  int imode;
  int gf_angle;
  uint32_t key0, key1;
  void* u;
  void* a;
  void* uf;
  void* af;
  void* g;   // gauge transform of the last tracked gauge fixing, [parity][site]
};

// mutable state shared by the chains of one context
struct CtxState {
  unsigned long long pass_ctr;    // Philox pass counter
  unsigned long long stream_pos;  // validation-stream position
  unsigned int status;            // LCE_STATUS_* bits
  unsigned int ticket;            // last-block ticket of the finalize kernel
  // the buffers of the reduce-behind blocks (lce_update.cu), set at context
  // creation: tile partials (slot i at rb_part + i * rb_slot_stride), the
  // chunk table of each tile table, chunk sums and totals
  const double* rb_part;
  unsigned long long rb_slot_stride;
  const int* rb_chunk_begin[4];
  double* rb_chunks;
  double* rb_totals;
};

// per-chain mutable state
struct ChainState {
  double delta;      // ahiggs1 step
  double gf_theta;   // last theta of the gauge fixing
  int gf_done;       // converged (or capped)
  int gf_iters;      // iterations done
  int gf_cap;        // iteration cap (<= 0: none)
  int gf_pad;
  unsigned int ticket;
  unsigned int pad2;
  double gf_limit;   // Fourier-accelerated fixing: theta to stop at
  double gf_step;    // Fourier-accelerated fixing: step gamma
};

// device status bits
enum : unsigned int {
  kStatusStreamExhausted = 1u,
  kStatusNaN = 2u,
  kStatusBarrierTimeout = 4u,
};

// grid barrier of the persistent sweep kernel (zeroed at context creation)
struct GridBar {
  unsigned count;  // arrivals, only ever incremented (wraps; compared as a difference)
  unsigned base;   // count at the start of the next launch
};
// polls of a grid barrier before the kernel gives up (>= 20 ns sleep each: >= 1.3 s)
constexpr unsigned kBarrierSpinLimit = 1u << 26;
constexpr int kPersistMinBlocks = 4;  // register cap 64 for the all-pass kernel
constexpr unsigned char kNoSlot = 0xff;

// one pass of a planned sweep
struct PlanEntry {
  unsigned char kind, eo, mu, slot;  // slot: reduction slot or kNoSlot
};

struct PassArgs {
  const ChainDev* chains;
  const int* blk_begin;   // nchains + 1 prefix of block counts
  CtxState* st;
  ChainState* cst;
  double* part;           // [block][kNQ] for this slot, or null
  const double* stream;   // validation stream (device) or null for Philox
  unsigned long long stream_n;
  unsigned long long stream_off;  // relative to st->stream_pos
  unsigned int pass_off;          // relative to st->pass_ctr
  int nchains;
  int eo;
  int fuse_renorm;
  int spt;                // sites per thread (a tile is bs * spt sites)
  int bs;                 // threads per block of the per-pass kernels
  int occ;                // resident threads per SM of the register cap (0: 4 x 256)
  // z-slab of a decomposed lattice (single-chain contexts): the passes visit
  // sites [s_lo, nh - s_lo) of each parity (the first and last planes are
  // halos), and site_off turns a site index into the whole lattice's for the
  // Philox counters; both 0 otherwise
  int s_lo, site_off;
  // validation stream: sites per parity of the whole lattice (a z-slab's
  // stream slots are the whole lattice's, at site s + site_off); 0: ch.nh
  int stream_nh;
  // programmatic dependent launch of the per-pass kernels.  rng_early: draw
  // the first site's uniforms before griddepcontrol.wait (the RNG counters,
  // written only by the finalize kernel, are settled for every pass but the
  // first of a queue).  trigger_late: let dependents launch only after this
  // kernel's wait (the first pass of a queue, so that no later pass can read
  // the counters while an earlier finalize still writes them).
  int rng_early, trigger_late;
  // reduce-behind: blocks [ntiles, gridDim.x) of a per-pass launch sum the
  // previous pass's tile partials (slot rb_slot & 0xff, tile table rb_slot >>
  // 8; the buffers in *st) into level-1 chunk sums (lce_update.cu), the same
  // additions in the same order as the finalize kernel's level 1, while this
  // pass's tiles update sites; rb_nitems = 0: no previous slot.  (Three ints
  // here: a larger argument block changed the register allocation of the
  // 64-register kernels.)
  int ntiles, rb_slot, rb_nitems;
};

struct FinalizeArgs {
  const ChainDev* chains;
  const int* blk_begin;
  CtxState* st;
  ChainState* cst;
  lce_meas* meas;         // [nchains]
  const double* part;     // slot i at part + i * slot_stride
  size_t slot_stride;
  double* totals;         // [nchains][kMaxSlots][kNQ]
  int nchains;
  int nslots;
  unsigned int npasses;           // advance of st->pass_ctr
  unsigned long long nstream;     // advance of st->stream_pos
  int single;                     // FP32 arithmetic for the ahiggs1 step update
  // two-level reduction of the tile partials (lce_update.cu): chunks of 128
  // tiles; chunk_begin = nchains + 1 prefix of chunks per chain
  const int* chunk_begin;
  double* chunks;                 // [chunk][kMaxSlots][kNQ]
  int nchunks;
  int ntiles0;                    // tiles of chain 0 (= blk_begin[1]), for the single-chain kernel
  // slots [0, pre) were summed to level-1 chunk sums by the pass after
  // theirs (reduce-behind); the finalize does level 1 of [pre, nslots) only
  int pre;
  unsigned char kinds[kMaxSlots];
  // the combine's routine groups (fin_groups), numbered by their last slot:
  // gid[i] = the group slot i belongs to (kNoGroup: none); gflags[g]:
  // kGrpHiggsLast (the last Higgs group: a2, a4, akin), kGrpKindLast (the
  // last group of its kind, or of {agauge, agauge1}: the kind's own
  // fields), kGrpMetro (an ahiggs1 group)
  // gbeg[g] / gend[g]: the first and the last slot of group g
  int ngroups, nmetro;
  unsigned char gid[kMaxSlots], gflags[kMaxSlots], gbeg[kMaxSlots], gend[kMaxSlots];
};
enum : unsigned char { kGrpHiggsLast = 1, kGrpKindLast = 2, kGrpMetro = 4, kNoGroup = 0xff };
void fin_groups(FinalizeArgs& f);

struct PersistArgs {
  PassArgs base;          // per-pass fields (eo, part, offsets) are filled in the kernel
  FinalizeArgs fin;
  GridBar* bar;
  int ntiles;             // tiles per pass (all chains)
  int npasses;
  PlanEntry plan[kMaxSlots];
  unsigned long long stream_off[kMaxSlots];
  unsigned short pass_off[kMaxSlots];  // Philox pass of each plan entry (3-hit passes take 3)
};

// ---- launchers (lce_update.cu)
template <typename R>
int persistent_grid();  // co-resident blocks of the persistent kernel on this device
template <typename R>
cudaError_t launch_persistent(const PersistArgs& a, int grid, cudaStream_t s);
template <typename R>
void launch_higgs(int mode, const PassArgs& a, int nblocks, cudaStream_t s);
template <typename R>
void launch_link(int mode, int mu, const PassArgs& a, int nblocks, cudaStream_t s);
void launch_finalize(const FinalizeArgs& f, cudaStream_t s);
// a sweep's first pass (ahiggs2, eo 0) with one extra block running the
// previous sweep's single-chain finalize fp (graphs of several sweeps)
template <typename R>
void launch_higgs_fin(const PassArgs& a, const FinalizeArgs& fp, int nblocks, cudaStream_t s);
template <typename R>
void launch_renorm(void* u, size_t nlinks, cudaStream_t s);
template <typename R>
void launch_debug_staple(const ChainDev* ch, int eo, int mu, double* out, int nh, cudaStream_t s);
template <typename R>
void launch_debug_force(const ChainDev* ch, int eo, double* out, int nh, cudaStream_t s);

// ---- field conversion (lce_fields.cu)
// reference order u[mu][eo][site(ld)][4], a[eo][site(ld)][3]  <->  device planes
template <typename Rin, typename R>
void launch_links_in(const Rin* src, void* dst, int nh, cudaStream_t s);
template <typename R, typename Rout>
void launch_links_out(const void* src, Rout* dst, int nh, cudaStream_t s);
template <typename Rin, typename R>
void launch_higgs_in(const Rin* src, void* dst, int nh, cudaStream_t s);
template <typename R, typename Rout>
void launch_higgs_out(const void* src, Rout* dst, int nh, cudaStream_t s);
template <typename R>
void launch_init_unit(void* u, void* a, int nh, double a3, cudaStream_t s);
template <typename R>
void launch_init_hot(void* u, void* a, int nh, uint32_t k0, uint32_t k1, cudaStream_t s);
void launch_flush(void* buf, size_t bytes, cudaStream_t s);

// ---- gauge fixing (lce_gaugefix.cu)
template <typename R>
void launch_gf_iteration(const ChainDev* ch, ChainState* cst, int track, double* part, int nh,
                         cudaStream_t s);
// one overrelaxed half-step over sites [s_lo, nh - s_lo) of local parity eo
// (a z-slab: s_lo = one plane); last: the second half-step, which writes the
// theta partials into part and reunitarises; track: also accumulate the
// transform G; returns the number of blocks (partials)
template <typename R>
int launch_gf_half(const ChainDev* ch, ChainState* cst, int eo, int last, double* part, int nh, int s_lo, int track,
                   cudaStream_t s);
// a half-step of f/it_gauge_fixing.f (reunitarising on the whole lattice's
// second half-step) on a z-slab's visited sites; returns the number of
// partials
template <typename R>
int launch_it_half(const ChainDev* ch, ChainState* cst, int eo, int last, double* part, int nh, int s_lo, int flags,
                   cudaStream_t s);
// convergence test of a z-slab decomposed fixing from the slabs' theta sums
void launch_gf_check_slabs(const ChainDev* ch, ChainState* cst, const double* sums, int nslabs, double nh,
                           cudaStream_t s, int fa = 0);
// one iteration of f/it_gauge_fixing.f (flags LCE_ITGF_*, step from cst->gf_step),
// then the convergence check of the overrelaxed form
template <typename R>
void launch_it_iteration(const ChainDev* ch, ChainState* cst, int flags, int renorm, double* part, int nh,
                         cudaStream_t s);
template <typename R>
void launch_gauge_apply(const ChainDev* ch, int nh, cudaStream_t s);
template <typename R>
void launch_transform_identity(void* g, int nh, cudaStream_t s);

// ---- Fourier-accelerated gauge fixing (lce_fourier.cu)
bool fa_supported(const ChainDev& ch);
// buffers for chains of up to vcap sites (fixed layout)
size_t fa_buffer_bytes(size_t vcap);
// fill the twiddle table of freshly allocated buffers
void fa_init_table(void* buf, size_t vcap, cudaStream_t s);
// one iteration; cst NULL (debug): never done, step gamma instead of the
// chain state's; cg: the conjugate-gradient form
template <typename R>
void launch_fa_iteration(const ChainDev* chd, const ChainDev& ch, ChainState* cst, double gamma, void* buf,
                         size_t vcap, double* part, double* omega_out, int track, bool with_check, bool with_apply,
                         bool cg, cudaStream_t s);
// the conjugate-gradient form starts its next iteration from the gradient
void fa_cg_reset(void* buf, size_t vcap, cudaStream_t s);
// the conjugate-gradient form on z-slabs: the whole lattice's CG state, F of
// this and the previous iteration ([2][2 fields][V] complex), the z
// transform's per-block pairs and one line-search triple per slab, on the
// first slab's device
struct FaSlabCg {
  void* cg;
  void* prev;
  double* pairs;
  double* tri;
  int nslabs;
  double nh_all;
};
// one stage of an iteration on a z-slab (lce_fourier.cu: 0 Delta and the x
// transforms into the whole lattice's buffer fft, returns the number of theta
// partials; 1 the y and z transforms of fft; 2 the inverse x transforms and
// g (CG: the direction); 3 g applied; CG: 4 the line derivatives (returns
// the number of partial triples), 5 the step from the slabs' sums, 6 g from
// the direction); Lg: the whole lattice; zl0, nzl, zg0, s_lo: the slab's
// visited planes and sites; cg: the CG form's whole-lattice buffers, or NULL
template <typename R>
int launch_fa_slab_stage(int stage, const ChainDev* chd, const ChainDev& ch, ChainState* cst, void* fft, void* buf,
                         size_t vcap, double* part, const int Lg[3], int zl0, int nzl, int zg0, int s_lo,
                         cudaStream_t s, const FaSlabCg* cg = nullptr);
// the CG state of a buffer, a reset of a state, its size; the direction
// field of a buffer ([component][parity][site] FP32)
void* fa_cg_state(void* buf, size_t vcap);
void fa_cg_reset_state(void* cg, cudaStream_t s);
size_t fa_cg_state_bytes();
void* fa_sdir_ptr(void* buf, size_t vcap);
// the per-block sums of a buffer (triples for up to vcap / 128 + 64 blocks)
double* fa_cgpart_ptr(void* buf, size_t vcap);
// the step transform g of a buffer ([parity][site], FP64 first rows)
void* fa_gstep_ptr(void* buf, size_t vcap);
// the first launch set-up failure of this host thread's Fourier kernels
// since the last call (kernel, line length, shared memory), or ""
std::string fa_take_error();
template <typename R>
void launch_gf_theta(const ChainDev* ch, double* part, int nh, cudaStream_t s);
void launch_sum_partials(const double* part, int nblocks, int nq, double* out, cudaStream_t s);

// ---- measurements (lce_meas.cu)
template <typename R>
void launch_slice_sums(const ChainDev* ch, int L3, double* slices, cudaStream_t s);
void launch_correlators(const double* slices, int L1, int L2, int L3, double* out, cudaStream_t s);
template <typename R>
void launch_plaquette(const ChainDev* ch, double* part, int nh, cudaStream_t s);
template <typename R>
void launch_functional(const ChainDev* ch, double* part, int nh, cudaStream_t s);

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// ---- learned warm start (lce_net.cu); all work on stream s
int net_device(lce_net* n);
// LCE_OK, or an error if a tensor-core kernel of the network gave up waiting
int net_status(lce_net* n);
// network input from the chain's U_f, A_f
int net_features(lce_net* n, const ChainDev* chd, const ChainDev& ch, bool f64, cudaStream_t s);
void net_predict(lce_net* n, const ChainDev& ch, cudaStream_t s);
// ch.g = Omega G_prev from the last prediction
int net_compose(lce_net* n, const ChainDev& ch, const void* gprev, bool f64, cudaStream_t s);
// record (last features, ch.g G_prev^+) as a training pair
int net_record(lce_net* n, const ChainDev& ch, const void* gprev, bool f64, cudaStream_t s);

// message returned by lce_last_error(NULL) on this host thread
void set_thread_error(const std::string& msg);

// Makes `device` current for the duration of one entry point and gives the
// caller back its own current device afterwards: a host thread may drive
// contexts (and networks) on several GPUs.  device < 0: nothing to do.
class DeviceScope {
 public:
  explicit DeviceScope(int device) {
    if (device < 0 || cudaGetDevice(&prev_) != cudaSuccess) return;
    if (prev_ != device && cudaSetDevice(device) == cudaSuccess) restore_ = true;
  }
  ~DeviceScope() {
    if (restore_) cudaSetDevice(prev_);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;

 private:
  int prev_ = -1;
  bool restore_ = false;
};

}  // namespace lce
