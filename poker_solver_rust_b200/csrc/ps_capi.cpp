// extern "C" boundary of the B200 range solver (include/ps_range_solver.h).
//
// A ps_batch owns N games packed into one device pool; a ps_game is a batch
// of one plus the navigation state of game/query.rs.  Host code here builds
// trees (ps_host.cpp), uploads them, launches the kernels of ps_kernels.cu and
// implements the query logic over the downloaded strategy / cfvalue arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ps_range_solver.h"
#include "ps_handeval.hpp"
#include "ps_host.hpp"
#include "ps_launch.hpp"

using namespace ps;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CU(x)                                                                           \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) return fail(PS_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---- per-device constants: hand table ----
// Every per-device cache below remembers the id of the CUDA context it was
// made in (current_context_id): a cudaDeviceReset destroys that context and
// everything allocated in it, so a cache from an older context is dropped
// (its memory is already gone) and made again in the current one.
struct DeviceConsts {
  int device = -1;
  unsigned long long ctx = 0;
  int32_t* table = nullptr;
  int nsm = 0;
  // The library's stream-ordered memory pool of the device: a batch's device
  // buffers come from it on the batch's stream and go back to it when the
  // batch ends, so building one batch while another solves neither waits for
  // the running kernels (as cudaMalloc / cudaFree do) nor maps memory anew.
  // Up to kPoolKeepBytes of freed memory stay in the pool for the next batch.
  cudaMemPool_t mpool = nullptr;
};
constexpr uint64_t kPoolKeepBytes = 8ull << 30;
constexpr int kMaxInstances = 4;  // spots per CTA in lockstep (ps_batch_opts.instances_per_cta) at most
// single games with at most this many acting hand-edges (sum over decision
// edges of the actor's hands) run on one thread-block cluster (Batch::build)
constexpr int64_t kClusterMaxEdgeHands = 131072;
std::mutex g_dev_mu;
std::mutex g_tune_mu;

struct CtxTag {  // where a cached allocation lives
  int dev = -1;
  unsigned long long ctx = 0;
};
cudaError_t current_tag(CtxTag* t) {
  cudaError_t e = cudaGetDevice(&t->dev);
  if (e != cudaSuccess) return e;
  return current_context_id(&t->ctx);
}

// Pinned host staging buffers, kept for reuse: a batch fills one, uploads it
// and hands it back, so back-to-back batches pay for page-locking once.  A
// buffer is reused only in the context that allocated it; buffers of an
// earlier context of the current device (ended by a device reset, which freed
// them) are forgotten.
struct PinnedPool {
  struct Buf {
    char* p;
    size_t bytes;
    CtxTag tag;
  };
  std::mutex mu;
  std::vector<Buf> free_;
  cudaError_t acquire(size_t bytes, char** out, CtxTag* tag) {
    cudaError_t e = current_tag(tag);
    if (e != cudaSuccess) return e;
    {
      std::lock_guard<std::mutex> lk(mu);
      free_.erase(std::remove_if(free_.begin(), free_.end(),
                                 [&](const Buf& b) { return b.tag.dev == tag->dev && b.tag.ctx != tag->ctx; }),
                  free_.end());
      for (size_t i = 0; i < free_.size(); ++i)
        if (free_[i].bytes >= bytes && free_[i].tag.ctx == tag->ctx) {
          *out = free_[i].p;
          free_.erase(free_.begin() + (long)i);
          return cudaSuccess;
        }
    }
    return cudaMallocHost(out, bytes);
  }
  void release(char* p, size_t bytes, const CtxTag& tag) {
    std::lock_guard<std::mutex> lk(mu);
    free_.push_back({p, bytes, tag});
    if (free_.size() > 2) {  // keep the two largest
      std::sort(free_.begin(), free_.end(), [](const Buf& a, const Buf& b) { return a.bytes > b.bytes; });
      CtxTag now;
      if (current_tag(&now) == cudaSuccess && now.ctx == free_.back().tag.ctx) cudaFreeHost(free_.back().p);
      free_.pop_back();
    }
  }
};
PinnedPool g_pinned;

// Streams and their four timing events, kept for reuse by the next batch:
// creating a stream or an event waits while a kernel of another batch runs
// (measured: 430 ms, the rest of a 600 ms solve), which would hold up
// building the next batch of a datagen job.  Reused only in the context that
// made them; at most kKeepStreams wait in the pool.
struct StreamPool {
  struct Entry {
    cudaStream_t s;
    cudaEvent_t ev[4];
    CtxTag tag;
  };
  static constexpr size_t kKeepStreams = 8;
  std::mutex mu;
  std::vector<Entry> free_;
  cudaError_t acquire(cudaStream_t* s, cudaEvent_t ev[4], CtxTag* made_in) {
    CtxTag& tag = *made_in;
    cudaError_t e = current_tag(&tag);
    if (e != cudaSuccess) return e;
    {
      std::lock_guard<std::mutex> lk(mu);
      // entries of an ended context of this device are gone with it
      free_.erase(std::remove_if(free_.begin(), free_.end(),
                                 [&](const Entry& x) { return x.tag.dev == tag.dev && x.tag.ctx != tag.ctx; }),
                  free_.end());
      for (size_t i = 0; i < free_.size(); ++i)
        if (free_[i].tag.dev == tag.dev && free_[i].tag.ctx == tag.ctx) {
          *s = free_[i].s;
          for (int k = 0; k < 4; ++k) ev[k] = free_[i].ev[k];
          free_.erase(free_.begin() + (long)i);
          return cudaSuccess;
        }
    }
    e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = cudaEventCreate(&ev[k]);
    return e;
  }
  // the stream's queued work (a batch's buffer frees) still runs in order.
  // made_in: the context acquire() found; a stream of a context that has
  // ended since (a device reset) is gone with it and is neither kept nor
  // destroyed
  void release(cudaStream_t s, cudaEvent_t ev[4], const CtxTag& made_in) {
    CtxTag tag;
    if (current_tag(&tag) != cudaSuccess) return;
    if (tag.dev != made_in.dev || tag.ctx != made_in.ctx) return;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (free_.size() < kKeepStreams && ev[0] && ev[1] && ev[2] && ev[3]) {
        Entry x{s, {ev[0], ev[1], ev[2], ev[3]}, tag};
        free_.push_back(x);
        return;
      }
    }
    for (int k = 0; k < 4; ++k)
      if (ev[k]) cudaEventDestroy(ev[k]);
    if (s) cudaStreamDestroy(s);
  }
};
StreamPool g_streams;


// Device staging for the per-call metadata of the datagen entry points
// (boards, pots, stacks, an error word): one buffer per device that only
// grows.  A call holds it, under the lock, until its stream work is done, so
// the common case allocates and frees nothing (cudaFree would synchronise the
// whole device).
struct DeviceStaging {
  std::mutex mu;
  char* buf[16] = {};
  size_t cap[16] = {};
  unsigned long long ctx[16] = {};
};
DeviceStaging g_staging;

// Holds the device's staging buffer until the lease ends.  A call that fails
// after it enqueued work on a stream waits for that stream (sync_on_release)
// before the buffer goes to the next call.
struct StagingLease {
  std::unique_lock<std::mutex> lk;
  char* ptr = nullptr;
  cudaStream_t pending = nullptr;
  bool busy = false;
  cudaError_t acquire(size_t bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
    unsigned long long ctx = 0;
    e = current_context_id(&ctx);
    if (e != cudaSuccess) return e;
    lk = std::unique_lock<std::mutex>(g_staging.mu);
    if (g_staging.ctx[dev] != ctx) {  // a buffer of an ended context is already freed
      g_staging.buf[dev] = nullptr;
      g_staging.cap[dev] = 0;
      g_staging.ctx[dev] = ctx;
    }
    if (g_staging.cap[dev] < bytes) {
      if (g_staging.buf[dev]) cudaFree(g_staging.buf[dev]);
      g_staging.buf[dev] = nullptr;
      g_staging.cap[dev] = 0;
      const size_t c = std::max<size_t>(bytes, (size_t)1 << 16);
      e = cudaMalloc(&g_staging.buf[dev], c);
      if (e != cudaSuccess) return e;
      g_staging.cap[dev] = c;
    }
    ptr = g_staging.buf[dev];
    return cudaSuccess;
  }
  // work that reads or writes the buffer is now queued on s
  void using_stream(cudaStream_t s) {
    pending = s;
    busy = true;
  }
  void done() { busy = false; }
  ~StagingLease() {
    if (busy) cudaStreamSynchronize(pending);  // an error path left copies in flight
  }
};
std::map<long, std::pair<int, int>> g_tune;  // autotuned (CTA size, scan-buffer warps) per
                                             // (device, hand-count class, tree-size class)
DeviceConsts g_dev[16];
std::map<long, std::array<int, 4>> g_flow_tune;  // autotuned dataflow shape (threads, scan buffers, spots per
                                                 // CTA, node parts) per (device, hand-count, tree-size class)

int device_consts(DeviceConsts** out) {
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 16) return fail(PS_ERR_CUDA, "device index out of range");
  unsigned long long ctx = 0;
  CU(current_context_id(&ctx));
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceConsts& d = g_dev[dev];
  if (d.ctx != ctx) d = DeviceConsts{};  // made in an ended context: its table is gone
  if (!d.table) {
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return fail(PS_ERR_CUDA, "the library is compiled for sm_100a (B200); found sm_" +
                                                       std::to_string(prop.major) + std::to_string(prop.minor));
    std::vector<int32_t> t(kHandTableSize + 64);
    int n = build_hand_table(t.data(), (int)t.size());
    if (n != kHandTableSize) return fail(PS_ERR_INVALID, "hand table size mismatch");
    CU(cudaMalloc(&d.table, sizeof(int32_t) * kHandTableSize));
    CU(cudaMemcpy(d.table, t.data(), sizeof(int32_t) * kHandTableSize, cudaMemcpyHostToDevice));
    cudaMemPoolProps pp = {};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = dev;
    CU(cudaMemPoolCreate(&d.mpool, &pp));
    uint64_t keep = kPoolKeepBytes;
    CU(cudaMemPoolSetAttribute(d.mpool, cudaMemPoolAttrReleaseThreshold, &keep));
    d.nsm = prop.multiProcessorCount;
    d.device = dev;
    d.ctx = ctx;
  }
  *out = &d;
  return PS_OK;
}

bool parse_tree_config(const ps_tree_config* c, TreeCfg& t, std::string& err) {
  t.initial_state = c->initial_state;
  if (t.initial_state < 0 || t.initial_state > 2) {
    err = "initial_state must be 0 (flop), 1 (turn) or 2 (river)";
    return false;
  }
  t.starting_pot = c->starting_pot;
  t.effective_stack = c->effective_stack;
  t.rake_rate = c->rake_rate;
  t.rake_cap = c->rake_cap;
  t.add_allin_threshold = c->add_allin_threshold;
  t.force_allin_threshold = c->force_allin_threshold;
  t.merging_threshold = c->merging_threshold;
  t.depth_limit = c->depth_limit;
  t.max_bets = c->max_bets;
  for (int s = 0; s < 3; ++s)
    for (int p = 0; p < 2; ++p) {
      const char* b = c->bet_sizes[s][p][0];
      const char* r = c->bet_sizes[s][p][1];
      if (!parse_menu(b ? b : "", false, t.menu[s][p].bet, err)) return false;
      if (!parse_menu(r ? r : "", true, t.menu[s][p].raise, err)) return false;
    }
  for (int k = 0; k < 2; ++k) {
    t.has_donk[k] = c->donk_sizes[k] != nullptr;
    if (t.has_donk[k] && !parse_menu(c->donk_sizes[k], false, t.donk[k], err)) return false;
  }
  return true;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

#ifndef PS_SINGLE_STAGE
#define PS_SINGLE_STAGE 1  // single games stage single-board tables in shared memory
#endif
#ifndef PS_SINGLE_BUFS
#define PS_SINGLE_BUFS 8  // single games: terminal scan buffers on all 8 warps
#endif

struct Layout {  // byte offsets inside the pool
  size_t cards[2], w[2], same[2], ops[2], steps[2], groups[2], nodes, board_cards, iso_perm[2], iso_off, iso_ent;  // static
  size_t gidx[2], coff[2], thr[2], nvalid[2], heads[2];                                                       // setup
  size_t R, S, SG, ipcfv, chcfv, rootv[2];                                                              // state
  size_t bcfv, breach;  // boundary values and boundary reach (kept across state resets)
};

// ---------------------------------------------------------------------------
// Batch: N games in one device pool
// ---------------------------------------------------------------------------
struct Batch {
  std::vector<std::unique_ptr<Game>> games;
  std::vector<Layout> lay;
  DeviceConsts* dc = nullptr;
  cudaStream_t stream = nullptr;
  char* pool = nullptr;
  size_t static_bytes = 0, setup_bytes = 0, state_bytes = 0, bnd_bytes = 0;
  char* h_static = nullptr;  // pinned staging of the static region (from g_pinned, during build only)
  size_t h_static_cap = 0;
  CtxTag h_static_tag;
  SpotDev* d_spots = nullptr;
  std::vector<SpotDev> h_spots;
  int2* d_work = nullptr;
  int nwork = 0;
  // boundary items: (spot, boundary ordinal) for every depth boundary of every
  // spot, spots in order, ordinals ascending
  std::vector<int2> items;
  int2* d_items = nullptr;
  bool ready = false;  // state zeroed and board tables built since the last reset
  char* adj_pool = nullptr;  // per-spot adjoint vectors (cotangents, weight and boundary gradients)
  char* rec_pool = nullptr;  // input ranges [n][2][1326] and RecordMeta [n] for the record writer
  size_t adj_bgrad_off = 0, adj_bytes = 0;
  float* d_scratch = nullptr;
  size_t scratch_floats = 0;
  int scratch_ctas = 0;
  Discount* d_disc = nullptr;
  int disc_cap = 0;
  float* d_target = nullptr;
  float* d_expl = nullptr;
  int* d_iters = nullptr;
  int* d_counter = nullptr;
  int* d_err = nullptr;
  int* d_order = nullptr;
  int inst_k = 1;            // spots per CTA solved in lockstep
  int ninst = 0;             // instances
  std::vector<int> inst;     // [ninst][inst_k] spot ids, -1 = empty
  int* d_inst = nullptr;
  int block = 256, grid = 1, ctas_per_sm = 0;
  int max_vstride = 32;
  SmemPlan plan{};
  int req_bufs = 0;  // scan buffers per CTA asked for (0 = one per warp)
  // grid mode: a single large spot runs on every CTA of a cooperative launch
  bool grid_mode = false;
  int grid_blocks = 0;
  int grid_cluster = 0;  // grid mode on the CTAs of one thread-block cluster (hardware barrier)
  unsigned* d_bar = nullptr;
  double* d_gred = nullptr;
  // dataflow scheduler (k_flow) for solve and run_iterations; the adjoint
  // and single spots keep the step-synchronous k_solve
  bool flow = false;
  int flow_block = 512, flow_grid = 0, flow_cps = 0, flow_lanes = 2, flow_parts = 1;
  SmemPlan flow_plan{};
  struct Trial {
    int block, bufs;
    float ms;
    int lanes = 0, parts = 0;  // dataflow trials: spots per CTA and node-op parts (0 = step-synchronous)
  };
  std::vector<Trial> tune_log;  // trials of the last autotune
  // dataflow shapes the sweep left within 6% of its best, re-timed by the
  // first fresh solve (refine_flow); empty when the choice is made
  std::vector<std::array<int, 4>> refine_cands;
  long refine_key = 0;
  int refine_cap = 0;
  std::vector<int> refine_order;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  CtxTag stream_tag;  // the context the stream and events were made in
  float last_solve_ms = 0, last_setup_ms = 0;
  std::vector<float> h_expl;
  std::vector<int> h_iters;

  // device buffers of the batch: from the device's pool, ordered on the
  // batch's stream (DeviceConsts::mpool)
  template <class T>
  cudaError_t dalloc(T** p, size_t bytes) {
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), std::max<size_t>(bytes, 1), dc->mpool, stream);
  }
  template <class T>
  void dfree(T*& p) {
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
  }

  ~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (h_static) g_pinned.release(h_static, h_static_cap, h_static_tag);
    if (stream) {  // the buffers go back to the pool behind the batch's last work
      dfree(pool);
      dfree(d_spots);
      dfree(d_work);
      dfree(d_items);
      dfree(adj_pool);
      dfree(rec_pool);
      dfree(d_scratch);
      dfree(d_disc);
      dfree(d_target);
      dfree(d_expl);
      dfree(d_bar);
      dfree(d_gred);
      dfree(d_iters);
      dfree(d_counter);
      dfree(d_err);
      dfree(d_order);
      dfree(d_inst);
    }
    if (stream) g_streams.release(stream, ev, stream_tag);
  }

  int build(const ps_batch_opts* opts) {
    int rc = device_consts(&dc);
    if (rc) return rc;
    CU(g_streams.acquire(&stream, ev, &stream_tag));
    const int n = (int)games.size();
    // a single game large enough for grid mode (below) evaluates all of a
    // pass's terminals in one step unless its caller chose the program
    // (ps_game_set_terminals_first): one long step per pass instead of one
    // per depth, each ended by a grid barrier
    {
      const char* env = std::getenv("PS_GRID_NODES");
      const long thr = env ? std::atol(env) : 16;
      if (n == 1 && games[0]->program_choice < 0 && thr > 0 && (long)games[0]->arena.size() >= thr &&
          !games[0]->terminals_first) {
        std::string err;
        if (!games[0]->recompile(true, err)) return fail(PS_ERR_INVALID, err);
      }
    }
    lay.resize(n);
    // ---- layout ----
    size_t so = 0, su = 0, st = 0, sb = 0;
    auto take = [](size_t& off, size_t bytes) {
      size_t r = off;
      off += align256(bytes);
      return r;
    };
    for (int i = 0; i < n; ++i) {
      Game& g = *games[i];
      Layout& L = lay[i];
      const size_t nb = g.boards.size();
      for (int p = 0; p < 2; ++p) {
        L.cards[p] = take(so, (size_t)g.H[p] * 2 + 16);
        L.w[p] = take(so, (size_t)g.hs[p] * 4);
        L.same[p] = take(so, (size_t)g.hs[p] * 2);
        L.ops[p] = take(so, g.prog[p].ops.size() * sizeof(Op));
        L.steps[p] = take(so, g.prog[p].steps.size() * sizeof(Step));
        L.groups[p] = take(so, g.prog[p].groups.size() * 2 + 16);
        L.iso_perm[p] = take(so, g.iso_perm[p].size() * (size_t)g.hs[p] * 2 + 16);
        L.gidx[p] = take(su, nb * 3 * g.hs[p] * 2);
        L.coff[p] = take(su, nb * 56 * 2);
        L.thr[p] = take(su, nb * g.hs[p] * kThrWords * 2);
        L.nvalid[p] = take(su, nb * 4);
        L.heads[p] = take(su, nb * 4 * (size_t)head_words(g.hs[p]));
      }
      L.nodes = take(so, g.arena.size() * sizeof(NodeDev));
      L.board_cards = take(so, nb * 5);
      L.iso_off = take(so, g.iso_list_off.size() * 4 + 16);
      L.iso_ent = take(so, g.iso_list.size() * 8 + 16);
      L.R = take(st, g.num_storage * 4 + 16);
      L.S = take(st, g.num_storage * 4 + 16);
      L.SG = take(st, g.num_storage * 4 + 16);  // strategy cache of the DCFR passes
      L.ipcfv = take(st, g.num_storage_ip * 4 + 16);
      L.chcfv = take(st, g.num_storage_chance * 4 + 16);
      for (int p = 0; p < 2; ++p) L.rootv[p] = take(st, (size_t)g.hs[p] * 4);
      L.bcfv = take(sb, (size_t)g.num_boundary * 2 * g.vstride * 4 + 16);
      L.breach = take(sb, (size_t)g.num_boundary * 2 * g.vstride * 4 + 16);
      max_vstride = std::max(max_vstride, g.vstride);
    }
    static_bytes = so;
    setup_bytes = su;
    state_bytes = st;
    bnd_bytes = sb;
    CU(dalloc(&pool, static_bytes + setup_bytes + state_bytes + bnd_bytes));
    // boundary values and reach start at zero.  Only batches with depth
    // boundaries clear them: the clear is a kernel, which cannot start while
    // another batch's solve holds every SM (measured: it held a datagen job's
    // next batch back by 430 ms of a 600 ms solve)
    bool any_boundary = false;
    for (const auto& gp : games) any_boundary = any_boundary || gp->num_boundary > 0;
    if (any_boundary) CU(cudaMemsetAsync(pool + static_bytes + setup_bytes + state_bytes, 0, bnd_bytes, stream));
    // the pinned staging buffer carries the static region and, after it, the
    // spot descriptors and the work, order, instance and boundary-item lists:
    // every upload then comes from pinned memory and is one asynchronous copy
    size_t nb_all = 0, bnd_all = 0;
    for (const auto& gp : games) {
      nb_all += gp->boards.size();
      bnd_all += (size_t)gp->num_boundary;
    }
    const size_t extra = align256(sizeof(SpotDev) * n) + align256(sizeof(int2) * nb_all) + align256(sizeof(int) * n) +
                         align256(sizeof(int) * (size_t)n * kMaxInstances) + align256(sizeof(int2) * bnd_all);
    h_static_cap = align256(std::max<size_t>(static_bytes, 16)) + extra;
    CU(g_pinned.acquire(h_static_cap, &h_static, &h_static_tag));
    // ---- fill static ----
    h_spots.resize(n);
    std::vector<int2> work;
    char* dS = pool;
    char* dU = pool + static_bytes;
    char* dT = pool + static_bytes + setup_bytes;
    char* dB = dT + state_bytes;
    // every spot fills its own regions: spread over the host cores
    auto fill = [&](int i) {
      Game& g = *games[i];
      Layout& L = lay[i];
      SpotDev& s = h_spots[i];
      std::memset(&s, 0, sizeof(s));
      for (int p = 0; p < 2; ++p) {
        uint8_t* cp = (uint8_t*)(h_static + L.cards[p]);
        for (int h = 0; h < g.H[p]; ++h) {
          cp[2 * h] = g.cards[p][h][0];
          cp[2 * h + 1] = g.cards[p][h][1];
        }
        float* wp = (float*)(h_static + L.w[p]);
        uint16_t* sp = (uint16_t*)(h_static + L.same[p]);
        for (int h = 0; h < g.hs[p]; ++h) {
          wp[h] = h < g.H[p] ? g.w[p][h] : 0.0f;
          sp[h] = h < g.H[p] ? g.same[p][h] : (uint16_t)0xFFFF;
        }
        std::memcpy(h_static + L.ops[p], g.prog[p].ops.data(), g.prog[p].ops.size() * sizeof(Op));
        std::memcpy(h_static + L.steps[p], g.prog[p].steps.data(), g.prog[p].steps.size() * sizeof(Step));
        std::memcpy(h_static + L.groups[p], g.prog[p].groups.data(), g.prog[p].groups.size() * 2);
        uint16_t* ip = (uint16_t*)(h_static + L.iso_perm[p]);
        for (size_t k = 0; k < g.iso_perm[p].size(); ++k)
          std::memcpy(ip + k * g.hs[p], g.iso_perm[p][k].data(), (size_t)g.hs[p] * 2);
        s.H[p] = g.H[p];
        s.hs[p] = g.hs[p];
        s.nsteps[p] = (int)g.prog[p].steps.size();
        s.root_slot[p] = g.prog[p].root_slot;
        s.cards[p] = (const uint8_t*)(dS + L.cards[p]);
        s.w[p] = (const float*)(dS + L.w[p]);
        s.same[p] = (const uint16_t*)(dS + L.same[p]);
        s.ops[p] = (const Op*)(dS + L.ops[p]);
        s.steps[p] = (const Step*)(dS + L.steps[p]);
        s.groups[p] = (const uint16_t*)(dS + L.groups[p]);
        s.iso_perm[p] = (const uint16_t*)(dS + L.iso_perm[p]);
        s.gidx[p] = (uint16_t*)(dU + L.gidx[p]);
        s.coff[p] = (uint16_t*)(dU + L.coff[p]);
        s.thr[p] = (uint16_t*)(dU + L.thr[p]);
        s.nvalid[p] = (int32_t*)(dU + L.nvalid[p]);
        s.heads[p] = (uint32_t*)(dU + L.heads[p]);
      }
      NodeDev* nd = (NodeDev*)(h_static + L.nodes);
      // reach scale of every node: the product of the rounded 1 / chance_factor
      // of the chance nodes above it, in the order the forward sweep applies them
      std::vector<float> pscale(g.arena.size(), 1.0f);
      for (size_t k = 0; k < g.arena.size(); ++k) {
        const ArenaNode& a = g.arena[k];
        if (a.terminal()) continue;
        const float f = a.chance() ? (float)(1.0f / (float)g.chance_factor(a)) : 1.0f;
        for (int ch = 0; ch < a.nch; ++ch) pscale[k + a.child_off + ch] = a.chance() ? pscale[k] * f : pscale[k];
      }
      for (size_t k = 0; k < g.arena.size(); ++k) {
        const ArenaNode& a = g.arena[k];
        NodeDev& d = nd[k];
        std::memset(&d, 0, sizeof(d));
        d.amount = a.amount;
        d.rs_off = a.rs_off;
        d.ip_off = a.ip_off;
        d.ch_off = a.ch_off;
        d.chance_factor = g.chance_factor(a);
        int sp = a.player & PL_MASK;
        d.ch_player = (a.chance() && (sp == 0 || sp == 1)) ? (sp ^ 1) : -1;
        d.boundary = g.bnd_ordinal[k];
        // evaluation.rs:64-68, :430 in f64, rounded once to f32
        double pot = (double)(g.cfg.starting_pot + 2 * a.amount);
        double half = 0.5 * pot;
        double rake = std::min(pot * g.cfg.rake_rate, g.cfg.rake_cap);
        d.amount_win = (float)((half - rake) / g.num_combinations);
        d.amount_lose = (float)(-half / g.num_combinations);
        d.amount_tie = (float)(-0.5 * rake / g.num_combinations);
        d.payoff_scale = (float)(half / g.num_combinations);
        d.path_scale = pscale[k];
      }
      uint8_t* bc = (uint8_t*)(h_static + L.board_cards);
      for (size_t b = 0; b < g.boards.size(); ++b) std::memcpy(bc + 5 * b, g.boards[b].data(), 5);
      std::memcpy(h_static + L.iso_off, g.iso_list_off.data(), g.iso_list_off.size() * 4);
      std::memcpy(h_static + L.iso_ent, g.iso_list.data(), g.iso_list.size() * 8);
      s.vstride = g.vstride;
      s.num_slots = g.num_slots;
      s.num_boards = (int)g.boards.size();
      s.starting_pot = g.cfg.starting_pot;
      s.raked = (g.cfg.rake_rate > 0.0 && g.cfg.rake_cap > 0.0) ? 1 : 0;
      s.num_boundary = g.num_boundary;
      s.num_combinations = g.num_combinations;
      s.rake_rate = g.cfg.rake_rate;
      s.rake_cap = g.cfg.rake_cap;
      s.nodes = (const NodeDev*)(dS + L.nodes);
      s.board_cards = (const uint8_t*)(dS + L.board_cards);
      s.iso_off = (const int32_t*)(dS + L.iso_off);
      s.iso_ent = (const int32_t*)(dS + L.iso_ent);
      s.bcfv = (const float*)(dB + L.bcfv);
      s.breach = g.num_boundary > 0 ? (float*)(dB + L.breach) : nullptr;
      for (int p = 0; p < 2; ++p) s.root_out[p] = (float*)(dT + L.rootv[p]);
      s.R = (float*)(dT + L.R);
      s.S = (float*)(dT + L.S);
      s.SG = (float*)(dT + L.SG);
      s.ipcfv = (float*)(dT + L.ipcfv);
      s.chcfv = (float*)(dT + L.chcfv);
    };
    {
      const int nt = std::max(1, std::min<int>(n / 64 + 1, std::min(16, (int)std::thread::hardware_concurrency())));
      std::vector<std::thread> th;
      for (int k = 0; k < nt; ++k)
        th.emplace_back([&, k] {
          for (int i = k; i < n; i += nt) fill(i);
        });
      for (auto& t : th) t.join();
    }
    for (int i = 0; i < n; ++i)
      for (size_t b = 0; b < games[i]->boards.size(); ++b) work.push_back(make_int2(i, (int)b));
    nwork = (int)work.size();
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < games[i]->num_boundary; ++k) items.push_back(make_int2(i, k));
    if (!items.empty()) CU(dalloc(&d_items, sizeof(int2) * items.size()));
    CU(dalloc(&d_spots, sizeof(SpotDev) * n));
    CU(dalloc(&d_work, sizeof(int2) * std::max(1, nwork)));
    CU(dalloc(&d_target, sizeof(float) * n));
    CU(dalloc(&d_expl, sizeof(float) * n));
    CU(dalloc(&d_iters, sizeof(int) * n));
    CU(dalloc(&d_counter, sizeof(int)));
    CU(dalloc(&d_err, sizeof(int)));
    CU(dalloc(&d_order, sizeof(int) * n));
    // launch configuration: warps per CTA (one op per warp at a time) and
    // whether single-board spots stage their board tables in shared memory
    int hs_max = 4;
    bool single_board = true;
    for (auto& gp : games) {
      hs_max = std::max(hs_max, std::max(gp->hs[0], gp->hs[1]));
      single_board &= gp->boards.size() == 1;
    }
    const bool tune = opts && opts->block_threads < 0;
    inst_k = opts && opts->instances_per_cta > 0 ? std::min(opts->instances_per_cta, kMaxInstances) : 1;
    req_bufs = opts ? opts->scan_buffers : 0;
    block = opts && opts->block_threads > 0 ? opts->block_threads : 256;
    block = std::max(64, std::min(256, (block / 32) * 32));
    const int stage = opts ? opts->stage_tables : -1;
    plan.vstride = max_vstride;
    plan.hs_max = hs_max;
    plan.warps = block / 32;
    plan.bufs = opts && opts->scan_buffers > 0 ? std::min(opts->scan_buffers, plan.warps)
                                               : std::max(1, plan.warps / 2);
    plan.tables = (single_board && stage == 1) ? table_bytes_for(hs_max, hs_max) : 0;
    plan.split = n <= dc->nsm ? 1 : 0;  // a CTA per spot with an SM to itself: latency-bound
    int occ = solve_occupancy(block, plan);
    ctas_per_sm = opts && opts->ctas_per_sm > 0 ? std::min(opts->ctas_per_sm, occ) : occ;
    grid = std::max(1, std::min(n, dc->nsm * ctas_per_sm));
    for (auto& gp : games) scratch_floats = std::max(scratch_floats, (size_t)gp->num_slots * gp->vstride);
    scratch_floats = (scratch_floats + 63) & ~(size_t)63;
    {
      const int sched = opts ? opts->scheduler : PS_SCHED_DEFAULT;
      if (sched < PS_SCHED_DEFAULT || sched > PS_SCHED_FLOW) return fail(PS_ERR_INVALID, "unknown scheduler");
      flow = sched == PS_SCHED_FLOW || (sched == PS_SCHED_DEFAULT && n > dc->nsm);
      if (flow) {
        int fb = opts && opts->flow_threads > 0 ? opts->flow_threads : 1024;
        fb = std::max(128, std::min(kMaxFlowThreads, (fb / 32) * 32));
        const int fl = opts && opts->flow_spots_per_cta > 0 ? opts->flow_spots_per_cta : 3;
        const int fp = opts && opts->node_parts > 0 ? opts->node_parts : 3;
        if (fl > kMaxFlowLanes || fp > 16) return fail(PS_ERR_INVALID, "flow_spots_per_cta 1..8, node_parts 1..16");
        const int rc = adopt_flow(fb, opts && opts->scan_buffers > 0 ? opts->scan_buffers : fb / 64, fl, fp,
                                  opts ? opts->ctas_per_sm : 0);
        if (rc) return rc;
      }
    }
    scratch_ctas = std::max(grid * inst_k, flow ? flow_grid * flow_lanes : 0);
    CU(dalloc(&d_scratch, sizeof(float) * scratch_floats * scratch_ctas));
    // a single tree of at least PS_GRID_NODES nodes (default 16; 0 = never)
    // is solved by all SMs at once: a lone game is latency-bound, and even a
    // 33-node river tree iterates 1.5x faster on every SM than on one
    {
      const char* env = std::getenv("PS_GRID_NODES");
      const long thr = env ? std::atol(env) : 16;
      if (n == 1 && thr > 0 && (long)games[0]->arena.size() >= thr) {
        const int gc = grid_ctas(block, plan);
        if (gc >= 2) {
          grid_mode = true;
          grid_blocks = gc;
          CU(dalloc(&d_bar, 64));
          CU(dalloc(&d_gred, 64));
          // A small tree runs on one cluster of 16 CTAs instead, its steps
          // ended by the hardware cluster barrier: a river game of 33 nodes
          // iterates 1.24x faster so, and datagen spots of 21-129 nodes solve
          // 1.21-1.41x faster; from about 150k acting hand-edges per iteration
          // the wider steps need the whole grid (a 141-node river tree with
          // 1081 hands ran 3% slower on the cluster, a 357-node one 24%).
          // PS_GRID_CLUSTER = C overrides: 0 = never, 2..16 = always, on C CTAs.
          const Game& g0 = *games[0];
          int64_t S = 0;
          for (const auto& nd : g0.arena)
            if (!nd.terminal() && !nd.chance()) S += (int64_t)nd.nch * g0.H[nd.player];
          const char* cl = std::getenv("PS_GRID_CLUSTER");
          const int want = cl ? std::atoi(cl) : (S <= kClusterMaxEdgeHands ? 16 : 0);
          if (want >= 2) {
            const int cc = grid_cluster_fits(std::min(want, 16), block, plan);
            if (cc >= 2) {
              grid_blocks = cc;
              grid_cluster = 1;
            }
          }
        }
      }
    }
    // order: largest estimated cost first (longest-processing-time first).
    // Work per iteration grows with the tree; the iterations to a target grow
    // with the stack-to-pot ratio (deeper stacks, more betting), which on the
    // datagen spots correlates 0.86 with the iteration count.
    std::vector<int> order(n);
    std::vector<double> cost(n);
    for (int i = 0; i < n; ++i) {
      order[i] = i;
      const Game& g = *games[i];
      const double spr = g.cfg.starting_pot > 0 ? (double)g.cfg.effective_stack / g.cfg.starting_pot : 1.0;
      cost[i] = ((double)g.num_storage + 4.0 * g.arena.size() * g.vstride) * std::log1p(std::max(spr, 0.05));
    }
    if (!opts || opts->sort_by_cost)
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    // instances: up to inst_k spots of one tree shape (and rake setting),
    // which share their step structure and are solved in lockstep by one CTA
    {
      std::map<std::string, std::vector<int>> by_shape;
      std::vector<std::string> shape_order;
      for (int i : order) {
        const Game& g = *games[i];
        std::string key;
        key.reserve(g.arena.size() * 3 + 8);
        for (const auto& a : g.arena) {
          key += (char)a.player;
          key += (char)(a.nch & 0xFF);
          key += (char)(a.nch >> 8);
        }
        key += (g.cfg.rake_rate > 0.0 && g.cfg.rake_cap > 0.0) ? 'r' : 'u';
        key += std::to_string(g.boards.size());
        auto& v = by_shape[key];
        if (v.empty()) shape_order.push_back(key);
        v.push_back(i);
      }
      std::vector<std::pair<double, std::vector<int>>> insts;
      for (const auto& key : shape_order) {
        const auto& v = by_shape[key];
        for (size_t j = 0; j < v.size(); j += inst_k) {
          std::vector<int> ids(inst_k, -1);
          double c = 0;
          for (int k = 0; k < inst_k && j + k < v.size(); ++k) {
            ids[k] = v[j + k];
            c += cost[v[j + k]];
          }
          insts.push_back({c, ids});
        }
      }
      if (!opts || opts->sort_by_cost)
        std::stable_sort(insts.begin(), insts.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
      ninst = (int)insts.size();
      inst.clear();
      for (auto& it : insts) inst.insert(inst.end(), it.second.begin(), it.second.end());
      CU(dalloc(&d_inst, sizeof(int) * std::max<size_t>(1, inst.size())));
    }
    // ---- upload (every source in the pinned staging buffer) ----
    if (inst.size() > (size_t)n * kMaxInstances) return fail(PS_ERR_INVALID, "instance list too long");
    char* hx = h_static + align256(std::max<size_t>(static_bytes, 16));
    auto put = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
      if (bytes == 0) return cudaSuccess;
      std::memcpy(hx, src, bytes);
      cudaError_t e = cudaMemcpyAsync(dst, hx, bytes, cudaMemcpyHostToDevice, stream);
      hx += align256(bytes);
      return e;
    };
    CU(cudaMemcpyAsync(pool, h_static, static_bytes, cudaMemcpyHostToDevice, stream));
    CU(put(d_spots, h_spots.data(), sizeof(SpotDev) * n));
    CU(put(d_work, work.data(), sizeof(int2) * nwork));
    CU(put(d_order, order.data(), sizeof(int) * n));
    CU(put(d_inst, inst.data(), sizeof(int) * inst.size()));
    CU(put(d_items, items.data(), sizeof(int2) * items.size()));
    CU(cudaStreamSynchronize(stream));
    g_pinned.release(h_static, h_static_cap, h_static_tag);  // uploaded: the staging buffer goes back to the pool
    h_static = nullptr;
    if (tune) return flow ? autotune_flow(order, opts ? opts->ctas_per_sm : 0) : autotune(order, opts ? opts->ctas_per_sm : 0);
    return PS_OK;
  }

  // Dataflow launch shape: CTAs of b threads with `bufs` scan-buffer warps,
  // `lanes` spots per CTA, node ops in `parts` column blocks, as many CTAs as
  // fit (at most cap_ctas per SM) but no more than the spots need.
  bool flow_shape(int b, int bufs, int lanes, int cap_ctas, int nspots, SmemPlan& pl, int& occ, int& g) const {
    pl = plan;
    pl.warps = b / 32;
    pl.bufs = std::max(1, std::min(pl.warps, bufs));
    pl.split = 0;
    occ = flow_occupancy(b, pl);
    if (occ < 1 || lanes > pl.warps) return false;
    if (cap_ctas > 0) occ = std::min(occ, cap_ctas);
    g = std::max(1, std::min((nspots + lanes - 1) / lanes, dc->nsm * occ));
    return true;
  }

  int adopt_flow(int b, int bufs, int lanes, int parts, int cap_ctas) {
    SmemPlan pl;
    int occ, g;
    if (!flow_shape(b, bufs, lanes, cap_ctas, (int)games.size(), pl, occ, g))
      return fail(PS_ERR_INVALID, "dataflow launch shape does not fit: " + std::to_string(b) + " threads, " +
                                      std::to_string(bufs) + " scan buffers, " + std::to_string(lanes) + " spots");
    if (d_scratch && (size_t)g * lanes > (size_t)scratch_ctas) {
      dfree(d_scratch);
      CU(dalloc(&d_scratch, sizeof(float) * scratch_floats * g * lanes));
      scratch_ctas = g * lanes;
    }
    flow_block = b;
    flow_plan = pl;
    flow_cps = occ;
    flow_grid = g;
    flow_lanes = lanes;
    flow_parts = parts;
    return PS_OK;
  }

  // Autotuner of the dataflow shape: times the real solve job (the reference
  // loop with its exploitability checks: one before the first iteration, after
  // the fifth and after the sixth) on a sample of the batch's spots taken
  // evenly from the cost order, for CTA sizes x scan buffers x spots per CTA x
  // node-op parts, and keeps the fastest.  The choice is cached per device and
  // tree-size class; the state the trials touched is cleared.
  int autotune_flow(const std::vector<int>& order, int cap_ctas) {
    const int n = (int)games.size();
    int hs_max = 4;
    double nodes = 0;
    for (auto& gp : games) {
      hs_max = std::max(hs_max, std::max(gp->hs[0], gp->hs[1]));
      nodes += (double)gp->arena.size();
    }
    const long key = (1l << 62) | ((long)dc->device << 40) | ((long)(req_bufs & 0xFF) << 32) |
                     ((long)(hs_max / 64) << 20) |
                     (long)std::min(1 << 19, (int)std::lround(std::log2(1.0 + nodes / n) * 4));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_flow_tune.find(key);
      if (it != g_flow_tune.end()) {
        const auto& c = it->second;
        return adopt_flow(c[0], c[1], c[2], c[3], cap_ctas);
      }
    }
    struct Cand {
      int b, bufs, lanes, parts;
    };
    std::vector<Cand> cands;
    for (int b : {256, 512, 1024})
      for (int lanes : {1, 2, 3, 4})
        for (int parts : {1, 2, 3}) {
          const int w = b / 32;
          if (req_bufs > 0) {
            cands.push_back({b, std::min(w, req_bufs), lanes, parts});
          } else {
            cands.push_back({b, std::max(1, w / 2), lanes, parts});
            cands.push_back({b, w, lanes, parts});
          }
        }
    int ns = 1;
    for (const auto& c : cands) {
      SmemPlan pl;
      int occ, g;
      if (flow_shape(c.b, c.bufs, c.lanes, cap_ctas, n, pl, occ, g)) ns = std::max(ns, g * c.lanes);
    }
    // the sweep's sample fills every candidate's lanes once; the refine runs
    // take kRefineWaves times as many spots, so lanes are rebound from the
    // queue as in a whole batch
    constexpr int kRefineWaves = 4;
    const int ns_sweep = std::min(n, ns);
    ns = std::min(n, kRefineWaves * ns);
    std::vector<SpotDev> sample(ns);
    std::vector<int> ids(ns);
    for (int i = 0; i < ns; ++i) {
      sample[i] = h_spots[order[(size_t)i * n / ns]];
      ids[i] = i;
    }
    // the sweep's spots: every kRefineWaves-th of the refine sample, so they
    // too are spread evenly over the cost order
    std::vector<int> sweep_ids(ns_sweep);
    for (int i = 0; i < ns_sweep; ++i) sweep_ids[i] = (int)((size_t)i * ns / ns_sweep);
    int rc = run_setup();
    if (rc) return rc;
    constexpr int kTrialIters = 6;
    if ((rc = ensure_disc(kTrialIters + 1))) return rc;
    size_t max_scr = 0;
    for (const auto& c : cands) {
      SmemPlan pl;
      int occ, g;
      if (flow_shape(c.b, c.bufs, c.lanes, cap_ctas, ns, pl, occ, g))
        max_scr = std::max(max_scr, (size_t)g * c.lanes);
    }
    char* tmp = nullptr;
    const size_t tb = align256(sizeof(SpotDev) * ns) + align256(20 * (size_t)ns) + 256;
    CU(cudaMalloc(&tmp, tb));
    std::unique_ptr<char, decltype(&cudaFree)> k1(tmp, &cudaFree);
    SpotDev* d_sample = (SpotDev*)tmp;
    int* d_ids = (int*)(tmp + align256(sizeof(SpotDev) * ns));  // the refine runs' queue: 0 .. ns-1
    int* d_sweep = d_ids + ns;                                   // the sweep's queue
    float* d_tz = (float*)(d_sweep + ns);    // targets 0: every sampled spot runs all trial iterations
    float* d_te = d_tz + ns;
    int* d_ti = (int*)(d_te + ns);
    int* d_cnt = (int*)(tmp + tb - 256);
    float* d_tscratch = nullptr;
    CU(cudaMalloc(&d_tscratch, sizeof(float) * scratch_floats * std::max<size_t>(1, max_scr)));
    std::unique_ptr<float, decltype(&cudaFree)> k2(d_tscratch, &cudaFree);
    CU(cudaMemcpyAsync(d_sample, sample.data(), sizeof(SpotDev) * ns, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_ids, ids.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_sweep, sweep_ids.data(), sizeof(int) * ns_sweep, cudaMemcpyHostToDevice, stream));
    CU(cudaMemsetAsync(d_tz, 0, sizeof(float) * ns, stream));
    const SolveJob job{0, kTrialIters, 1, 0};
    // one trial: a warm-up run, then the timed run (device ms)
    auto trial = [&](const Cand& c, const SolveJob& jb, const int* q, int nq, float* out_ms,
                     int* out_bufs) -> cudaError_t {
      SmemPlan pl;
      int occ, g;
      *out_ms = 0.f;
      if (!flow_shape(c.b, c.bufs, c.lanes, cap_ctas, nq, pl, occ, g)) return cudaSuccess;
      cudaError_t e = cudaSuccess;
      for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
        e = cudaMemsetAsync(d_cnt, 0, sizeof(int), stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2], stream);
        if (e == cudaSuccess)
          e = launch_flow(d_sample, nq, q, d_cnt, d_disc, jb, d_tz, d_tscratch, scratch_floats, d_te, d_ti, d_err,
                          g, c.b, c.lanes, c.parts, pl, stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[3], stream);
      }
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e == cudaSuccess) e = cudaEventElapsedTime(out_ms, ev[2], ev[3]);
      *out_bufs = pl.bufs;
      return e;
    };
    Cand best{flow_block, flow_plan.bufs, flow_lanes, flow_parts};
    float best_ms = 0;
    std::vector<std::pair<float, Cand>> swept;
    for (const auto& c : cands) {
      float ms = 0;
      int bufs = 0;
      CU(trial(c, job, d_sweep, ns_sweep, &ms, &bufs));
      if (ms <= 0.f) continue;
      tune_log.push_back(Trial{c.b, bufs, ms, c.lanes, c.parts});
      swept.push_back({ms, Cand{c.b, bufs, c.lanes, c.parts}});
      if (best_ms == 0 || ms < best_ms) {
        best_ms = ms;
        best = {c.b, bufs, c.lanes, c.parts};
      }
    }
    // refine: the shapes within 6% of the sweep's best (at most 6) run again at
    // the batch's first solve, on a larger sample with the solve's own targets
    // and iteration limit (refine_flow); until then the sweep's best stands
    refine_cands.clear();
    if (ns > ns_sweep && !swept.empty()) {
      std::stable_sort(swept.begin(), swept.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      for (size_t i = 0; i < swept.size() && i < 6 && swept[i].first <= 1.06f * best_ms; ++i) {
        const Cand& c = swept[i].second;
        refine_cands.push_back({c.b, c.bufs, c.lanes, c.parts});
      }
      if (refine_cands.size() < 2) refine_cands.clear();
    }
    if ((rc = check_err())) return rc;
    if (refine_cands.empty()) {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_flow_tune[key] = {best.b, best.bufs, best.lanes, best.parts};
    } else {
      refine_key = key;
      refine_cap = cap_ctas;
      refine_order = order;
    }
    CU(cudaMemsetAsync(pool + static_bytes + setup_bytes, 0, state_bytes, stream));
    ready = true;  // the trials' state is cleared and the board tables stay built
    rc = adopt_flow(best.b, best.bufs, best.lanes, best.parts, cap_ctas);
    if (rc) return rc;
    CU(cudaStreamSynchronize(stream));
    return PS_OK;
  }

  // The autotuner's refine stage, run by the batch's first fresh solve: each
  // shape the sweep left within 6% of its best solves a sample of the batch
  // (four waves of spots, evenly along the cost order) from zero state with
  // the solve's own targets and iteration limit, as the whole batch will, so
  // the spots' spread of iteration counts and the lanes' rebinding count in
  // the timing.  The fastest is adopted and cached; the trials are logged
  // after the sweep's.  The state is zeroed again afterwards.
  int refine_flow(uint32_t max_iter, const float* target) {
    const int n = (int)games.size();
    int ns = 1;
    for (const auto& c : refine_cands) {
      SmemPlan pl;
      int occ, g;
      if (flow_shape(c[0], c[1], c[2], refine_cap, n, pl, occ, g)) ns = std::max(ns, g * c[2]);
    }
    size_t max_scr = (size_t)ns;
    ns = std::min(n, 4 * ns);
    std::vector<SpotDev> sample(ns);
    std::vector<int> ids(ns);
    std::vector<float> tg(ns);
    for (int i = 0; i < ns; ++i) {
      const int k = refine_order[(size_t)i * n / ns];
      sample[i] = h_spots[k];
      ids[i] = i;
      tg[i] = target[k];
    }
    char* tmp = nullptr;
    const size_t tb = align256(sizeof(SpotDev) * ns) + align256(16 * (size_t)ns) + 256;
    CU(cudaMalloc(&tmp, tb));
    std::unique_ptr<char, decltype(&cudaFree)> k1(tmp, &cudaFree);
    SpotDev* d_sample = (SpotDev*)tmp;
    int* d_ids = (int*)(tmp + align256(sizeof(SpotDev) * ns));
    float* d_tg = (float*)(d_ids + ns);
    float* d_te = d_tg + ns;
    int* d_ti = (int*)(d_te + ns);
    int* d_cnt = (int*)(tmp + tb - 256);
    float* d_tscratch = nullptr;
    CU(cudaMalloc(&d_tscratch, sizeof(float) * scratch_floats * max_scr));
    std::unique_ptr<float, decltype(&cudaFree)> k2(d_tscratch, &cudaFree);
    CU(cudaMemcpyAsync(d_sample, sample.data(), sizeof(SpotDev) * ns, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_ids, ids.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(d_tg, tg.data(), sizeof(float) * ns, cudaMemcpyHostToDevice, stream));
    const SolveJob job{0, (int)max_iter, 1, 0};
    std::array<int, 4> best = refine_cands[0];
    float best_ms = 0;
    for (const auto& c : refine_cands) {
      SmemPlan pl;
      int occ, g;
      if (!flow_shape(c[0], c[1], c[2], refine_cap, ns, pl, occ, g)) continue;
      CU(cudaMemsetAsync(pool + static_bytes + setup_bytes, 0, state_bytes, stream));
      CU(cudaMemsetAsync(d_cnt, 0, sizeof(int), stream));
      CU(cudaEventRecord(ev[2], stream));
      CU(launch_flow(d_sample, ns, d_ids, d_cnt, d_disc, job, d_tg, d_tscratch, scratch_floats, d_te, d_ti, d_err, g,
                     c[0], c[2], c[3], pl, stream));
      CU(cudaEventRecord(ev[3], stream));
      CU(cudaStreamSynchronize(stream));
      float ms = 0;
      CU(cudaEventElapsedTime(&ms, ev[2], ev[3]));
      tune_log.push_back(Trial{c[0], pl.bufs, ms, c[2], c[3]});
      if (best_ms == 0 || ms < best_ms) {
        best_ms = ms;
        best = {c[0], pl.bufs, c[2], c[3]};
      }
    }
    int rc = check_err();
    if (rc) return rc;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_flow_tune[refine_key] = best;
    }
    refine_cands.clear();
    refine_order.clear();
    CU(cudaMemsetAsync(pool + static_bytes + setup_bytes, 0, state_bytes, stream));
    return adopt_flow(best[0], best[1], best[2], best[3], refine_cap);
  }

  // A first call other than a fresh solve keeps the sweep's choice: it is
  // cached as it stands, so the next batch of the class does not sweep again.
  void settle_tune() {
    if (refine_cands.empty()) return;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_flow_tune[refine_key] = {flow_block, flow_plan.bufs, flow_lanes, flow_parts};
    refine_cands.clear();
    refine_order.clear();
  }

  // The batch's solve-type job (iterations, checks, epilogue) on every spot,
  // with the scheduler the batch runs.
  cudaError_t launch_job(const SolveJob& job) {
    if (flow)
      return launch_flow(d_spots, (int)games.size(), d_order, d_counter, d_disc, job, d_target, d_scratch,
                         scratch_floats, d_expl, d_iters, d_err, flow_grid, flow_block, flow_lanes, flow_parts,
                         flow_plan, stream);
    return launch_solve(d_spots, ninst, inst_k, d_inst, d_counter, d_disc, job, d_target, d_scratch, scratch_floats,
                        d_expl, d_iters, d_err, grid, block, plan, stream);
  }

  // Launch shape for a CTA of `b` threads: shared-memory plan, CTAs per SM
  // and grid for `nspots` spots.
  void shape_for(int b, int bufs, int cap_ctas, int nspots, SmemPlan& pl, int& occ, int& g) const {
    pl = plan;
    pl.warps = b / 32;
    pl.bufs = std::max(1, std::min(pl.warps, bufs));
    occ = solve_occupancy(b, pl);
    if (cap_ctas > 0) occ = std::min(occ, cap_ctas);
    g = std::max(1, std::min(nspots, dc->nsm * occ));
  }

  // Autotuner: times a fixed amount of work (a few DCFR iterations of a
  // sample of this batch's spots, taken evenly from the cost order) with every
  // CTA size from 64 to the compiled maximum in steps of one warp, each with
  // as many CTAs as fit, and keeps the fastest.  The choice is cached per
  // device and tree-size class, and the state the trial runs touched is
  // cleared afterwards.
  int autotune(const std::vector<int>& order, int cap_ctas) {
    const int n = (int)games.size();
    int hs_max = 4;
    double nodes = 0;
    for (auto& gp : games) {
      hs_max = std::max(hs_max, std::max(gp->hs[0], gp->hs[1]));
      nodes += (double)gp->arena.size();
    }
    const long key = ((long)dc->device << 40) | ((long)(req_bufs & 0xFF) << 32) | ((long)(hs_max / 64) << 20) |
                     (long)std::min(1 << 19, (int)std::lround(std::log2(1.0 + nodes / n) * 4));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) return adopt_block(it->second.first, it->second.second, cap_ctas);
    }
    // candidates: CTA size x warps that own a terminal scan buffer (half or
    // all of them, or the count the caller fixed)
    std::vector<std::pair<int, int>> cands;
    for (int b = 128; b <= kMaxSolveBlock; b += 32) {
      const int w = b / 32;
      if (req_bufs > 0) {
        cands.push_back({b, std::min(w, req_bufs)});
      } else {
        cands.push_back({b, std::max(1, w / 2)});
        cands.push_back({b, w});
      }
    }
    int max_grid = 1;
    for (auto [b, nb] : cands) {
      SmemPlan pl;
      int occ, g;
      shape_for(b, nb, cap_ctas, n, pl, occ, g);
      max_grid = std::max(max_grid, g);
    }
    const int ns = std::min(n, max_grid);
    std::vector<SpotDev> sample(ns);
    for (int i = 0; i < ns; ++i) sample[i] = h_spots[order[(size_t)i * n / ns]];
    int rc = run_setup();
    if (rc) return rc;
    if ((rc = ensure_disc(16))) return rc;
    SpotDev* d_sample = nullptr;
    float* d_tscratch = nullptr;
    CU(cudaMalloc(&d_sample, sizeof(SpotDev) * ns));
    std::unique_ptr<SpotDev, decltype(&cudaFree)> k1(d_sample, &cudaFree);
    CU(cudaMalloc(&d_tscratch, sizeof(float) * scratch_floats * ns));
    std::unique_ptr<float, decltype(&cudaFree)> k2(d_tscratch, &cudaFree);
    CU(cudaMemcpyAsync(d_sample, sample.data(), sizeof(SpotDev) * ns, cudaMemcpyHostToDevice, stream));
    std::pair<int, int> best{block, plan.bufs};
    float best_ms = 0;
    for (auto [b, nb] : cands) {
      SmemPlan pl;
      int occ, g;
      shape_for(b, nb, cap_ctas, ns, pl, occ, g);
      CU(launch_iterate(d_sample, ns, d_disc, 0, 2, d_tscratch, scratch_floats, d_err, g, b, pl, stream));
      CU(cudaEventRecord(ev[2], stream));
      CU(launch_iterate(d_sample, ns, d_disc, 2, 8, d_tscratch, scratch_floats, d_err, g, b, pl, stream));
      CU(cudaEventRecord(ev[3], stream));
      CU(cudaStreamSynchronize(stream));
      float ms = 0;
      CU(cudaEventElapsedTime(&ms, ev[2], ev[3]));
      tune_log.push_back({b, nb, ms});
      if (best_ms == 0 || ms < best_ms) {
        best_ms = ms;
        best = {b, nb};
      }
    }
    if ((rc = check_err())) return rc;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune[key] = best;
    }
    CU(cudaMemsetAsync(pool + static_bytes + setup_bytes, 0, state_bytes, stream));
    ready = true;  // the trials' state is cleared and the board tables stay built
    return adopt_block(best.first, best.second, cap_ctas);
  }

  // Switches the batch to CTAs of `b` threads with `bufs` scan-buffer warps
  // (scratch sized for the new grid).
  int adopt_block(int b, int bufs, int cap_ctas) {
    const int n = (int)games.size();
    SmemPlan pl;
    int occ, g;
    shape_for(b, bufs, cap_ctas, n, pl, occ, g);
    if (g * inst_k > scratch_ctas) {
      dfree(d_scratch);
      CU(dalloc(&d_scratch, sizeof(float) * scratch_floats * g * inst_k));
      scratch_ctas = g * inst_k;
    }
    block = b;
    plan = pl;
    ctas_per_sm = occ;
    grid = g;
    CU(cudaStreamSynchronize(stream));
    return PS_OK;
  }

  // One grid-mode launch of this batch's single spot.
  cudaError_t grid_launch(const GridJob& job) {
    return launch_grid(d_spots, job, d_disc, d_scratch, scratch_floats, d_expl, d_iters, d_bar, d_gred, d_err,
                       grid_blocks, block, plan, stream, grid_cluster);
  }

  // Average-strategy pass(es) of the single spot: on every SM in grid mode,
  // on one CTA otherwise (k_average).
  cudaError_t average(int save, int player, const float* root_reach, float* out, int owner, float* bgrad,
                      float* breach = nullptr) {
    if (grid_mode)
      return grid_launch(
          {save ? GRID_FINALIZE : GRID_AVERAGE, 0, 0, 0.f, player, owner, root_reach, bgrad, out, breach});
    return launch_average(d_spots, 1, save, player, root_reach, d_scratch, scratch_floats, out, d_err, 1, block, plan,
                          stream, owner, bgrad, breach);
  }

  // Zeroes the solver state and rebuilds the per-board tables on the device.
  int enqueue_setup() {
    CU(cudaMemsetAsync(pool + static_bytes + setup_bytes, 0, state_bytes, stream));
    CU(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    CU(launch_setup(d_spots, d_work, nwork, dc->table, d_err, std::max(1, std::min(nwork, dc->nsm * 4)), stream));
    ready = true;
    return PS_OK;
  }

  int run_setup() {
    int rc = enqueue_setup();
    if (rc) return rc;
    CU(cudaStreamSynchronize(stream));
    return check_err();
  }

  int check_err() {
    int e = 0;
    CU(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    if (e) return fail(PS_ERR_DEVICE, "kernel error flag " + std::to_string(e));
    return PS_OK;
  }

  int ensure_disc(uint32_t upto) {
    if ((int)upto <= disc_cap) return PS_OK;
    int cap = std::max<int>(upto, std::max(1024, 2 * disc_cap));
    std::vector<Discount> h(cap);
    for (int t = 0; t < cap; ++t) h[t] = discount_params((uint32_t)t);
    dfree(d_disc);
    CU(dalloc(&d_disc, sizeof(Discount) * cap));
    CU(cudaMemcpyAsync(d_disc, h.data(), sizeof(Discount) * cap, cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));  // h is released on return
    disc_cap = cap;
    return PS_OK;
  }

  // fresh = true: a complete job (state reset + board setup + solve), timed
  // as setup_ms + solve_ms; fresh = false continues from the current state.
  int solve(uint32_t max_iter, const float* target, bool fresh) {
    const int n = (int)games.size();
    int rc = ensure_disc(max_iter + 1);
    if (rc) return rc;
    if (grid_mode) {
      if (fresh && (rc = run_setup())) return rc;
      CU(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
      CU(cudaEventRecord(ev[2], stream));
      GridJob job{GRID_SOLVE, 0, (int)max_iter, target[0], 0, -1, nullptr, nullptr, nullptr};
      CU(launch_grid(d_spots, job, d_disc, d_scratch, scratch_floats, d_expl, d_iters, d_bar, d_gred, d_err,
                     grid_blocks, block, plan, stream, grid_cluster));
      CU(cudaEventRecord(ev[3], stream));
      h_expl.resize(1);
      h_iters.resize(1);
      CU(cudaMemcpyAsync(h_expl.data(), d_expl, sizeof(float), cudaMemcpyDeviceToHost, stream));
      CU(cudaMemcpyAsync(h_iters.data(), d_iters, sizeof(int), cudaMemcpyDeviceToHost, stream));
      CU(cudaStreamSynchronize(stream));
      CU(cudaEventElapsedTime(&last_solve_ms, ev[2], ev[3]));
      last_setup_ms = 0;
      return check_err();
    }
    if (fresh && flow && !refine_cands.empty() && (rc = refine_flow(max_iter, target))) return rc;
    settle_tune();
    CU(cudaMemcpyAsync(d_target, target, sizeof(float) * n, cudaMemcpyHostToDevice, stream));
    CU(cudaMemsetAsync(d_counter, 0, sizeof(int), stream));
    CU(cudaEventRecord(ev[1], stream));
    if (fresh && (rc = enqueue_setup())) return rc;
    if (!fresh) CU(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    CU(cudaEventRecord(ev[2], stream));
    const SolveJob job{0, (int)max_iter, 1, EPI_ROOT};
    CU(launch_job(job));
    CU(cudaEventRecord(ev[3], stream));
    h_expl.resize(n);
    h_iters.resize(n);
    CU(cudaMemcpyAsync(h_expl.data(), d_expl, sizeof(float) * n, cudaMemcpyDeviceToHost, stream));
    CU(cudaMemcpyAsync(h_iters.data(), d_iters, sizeof(int) * n, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    CU(cudaEventElapsedTime(&last_solve_ms, ev[2], ev[3]));
    CU(cudaEventElapsedTime(&last_setup_ms, ev[1], ev[2]));
    return check_err();
  }

  // Board size shared by every spot (records of one file share it), or -1.
  int board_size() const {
    int bs = -1;
    for (auto& gp : games) {
      const int k = gp->turn == NOT_DEALT ? 3 : gp->river == NOT_DEALT ? 4 : 5;
      if (bs >= 0 && k != bs) return -1;
      bs = k;
    }
    return bs;
  }

  size_t record_bytes() const {
    const int bs = board_size();
    return bs < 0 ? 0 : games.size() * 2 * (size_t)(1 + bs + 13 + 13 * 1326);
  }

  // Packs the training records of every spot into `out` (device memory).
  int records(uint8_t* out) {
    const int n = (int)games.size();
    if (board_size() < 0) return fail(PS_ERR_INVALID, "records of one batch need one board size");
    const size_t rb = align256((size_t)n * 2 * 1326 * 4);
    if (!rec_pool) {
      std::vector<float> r((size_t)n * 2 * 1326);
      std::vector<RecordMeta> m(n);
      for (int i = 0; i < n; ++i) {
        const Game& g = *games[i];
        std::memcpy(&r[(size_t)i * 2 * 1326], g.range[0], 4 * 1326);
        std::memcpy(&r[(size_t)i * 2 * 1326 + 1326], g.range[1], 4 * 1326);
        RecordMeta& x = m[i];
        std::memset(&x, 0, sizeof(x));
        x.pot = (float)g.cfg.starting_pot;
        x.stack = (float)g.cfg.effective_stack;
        const uint8_t bd[5] = {g.flop[0], g.flop[1], g.flop[2], g.turn, g.river};
        x.board_size = (uint8_t)(g.turn == NOT_DEALT ? 3 : g.river == NOT_DEALT ? 4 : 5);
        std::memcpy(x.board, bd, x.board_size);
      }
      CU(dalloc(&rec_pool, rb + sizeof(RecordMeta) * n));
      CU(cudaMemcpyAsync(rec_pool, r.data(), 4 * r.size(), cudaMemcpyHostToDevice, stream));
      CU(cudaMemcpyAsync(rec_pool + rb, m.data(), sizeof(RecordMeta) * n, cudaMemcpyHostToDevice, stream));
    }
    CU(launch_pack_records(d_spots, n, (const float*)rec_pool, (const RecordMeta*)(rec_pool + rb), out, stream));
    CU(cudaStreamSynchronize(stream));
    return PS_OK;
  }

  // Allocates the per-spot adjoint vectors on first use: cotangents and
  // weight gradients [hs] per player, then all boundary gradients.
  int ensure_adjoint() {
    if (adj_pool) return PS_OK;
    const int n = (int)games.size();
    size_t off = 0;
    std::vector<size_t> o(n);
    for (int i = 0; i < n; ++i) {
      o[i] = off;
      off += align256(16 * (size_t)(games[i]->hs[0] + games[i]->hs[1]));
    }
    adj_bgrad_off = off;
    std::vector<size_t> ob(n);
    for (int i = 0; i < n; ++i) {
      ob[i] = off;
      off += align256((size_t)games[i]->num_boundary * 2 * games[i]->vstride * 4);
    }
    adj_bytes = std::max<size_t>(off, 256);
    CU(dalloc(&adj_pool, adj_bytes));
    for (int i = 0; i < n; ++i) {
      SpotDev& s = h_spots[i];
      float* v = (float*)(adj_pool + o[i]);
      const int h0 = games[i]->hs[0], h1 = games[i]->hs[1];
      s.adj_g[0] = v;
      s.adj_g[1] = v + h0;
      s.adj_dw[0] = v + h0 + h1;
      s.adj_dw[1] = v + 2 * h0 + h1;
      s.bgrad = games[i]->num_boundary > 0 ? (float*)(adj_pool + ob[i]) : nullptr;
    }
    CU(cudaMemcpyAsync(d_spots, h_spots.data(), sizeof(SpotDev) * n, cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return PS_OK;
  }

  // Fixed-strategy evaluation under the average strategy and its adjoint for
  // every spot from the cotangents already in sp.adj_g: root values into
  // sp.root_out, gradients into sp.adj_dw and sp.bgrad.
  int adjoint() {
    for (auto& gp : games)
      if (!gp->iso_list.empty())
        return fail(PS_ERR_UNSUPPORTED, "the adjoint needs spots without isomorphic chance pruning");
    int rc = ensure_adjoint();
    if (rc) return rc;
    if (!ready && (rc = enqueue_setup())) return rc;
    CU(cudaMemsetAsync(adj_pool + adj_bgrad_off, 0, adj_bytes - adj_bgrad_off, stream));
    CU(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    if (grid_mode) {
      const SpotDev& s = h_spots[0];
      for (int pass = 0; pass < 4; ++pass) {
        const int p = pass < 2 ? pass : 3 - pass;
        CU(average(0, p, pass < 2 ? s.w[p ^ 1] : s.adj_g[p ^ 1], pass < 2 ? s.root_out[p] : s.adj_dw[p],
                   pass < 2 ? -1 : (p ^ 1), s.bgrad));
      }
    } else {
      CU(cudaMemsetAsync(d_counter, 0, sizeof(int), stream));
      SolveJob job{0, 0, 0, 0};
      job.adjoint = 1;
      CU(launch_solve(d_spots, ninst, inst_k, d_inst, d_counter, d_disc, job, d_target, d_scratch, scratch_floats,
                      d_expl, d_iters, d_err, grid, block, plan, stream));
    }
    CU(cudaStreamSynchronize(stream));
    return check_err();
  }

  // DCFR iterations [t0, t1) of every spot from the current state, with no
  // exploitability checks (batch.rs:414-535 run_iterations), then the
  // requested epilogue (EPI_ROOT: root cfvalues and boundary reach under the
  // average strategy; EPI_EXPL: exploitability, reported by ps_batch_results
  // with iterations = t1).  The first call after construction or a reset
  // zeroes the state and builds the board tables.
  int run_iterations(uint32_t t0, uint32_t t1, int epilogue) {
    settle_tune();
    const int n = (int)games.size();
    int rc = ensure_disc(t1 + 1);
    if (rc) return rc;
    if (!ready && (rc = enqueue_setup())) return rc;
    CU(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    CU(cudaEventRecord(ev[2], stream));
    if (grid_mode) {
      CU(grid_launch({GRID_ITERATE, (int)t0, (int)t1, 0.f, 0, -1, nullptr, nullptr, nullptr}));
      if (epilogue & EPI_EXPL) CU(grid_launch({GRID_EXPL, 0, 0, 0.f, 0, -1, nullptr, nullptr, nullptr}));
      if (epilogue & EPI_ROOT)
        for (int p = 0; p < 2; ++p)
          CU(grid_launch({GRID_AVERAGE, 0, 0, 0.f, p, -1, nullptr, nullptr, h_spots[0].root_out[p],
                          h_spots[0].breach}));
    } else {
      CU(cudaMemsetAsync(d_counter, 0, sizeof(int), stream));
      const SolveJob job{(int)t0, (int)t1, 0, epilogue};
      CU(launch_job(job));
    }
    CU(cudaEventRecord(ev[3], stream));
    if (epilogue & EPI_EXPL) {
      h_expl.resize(n);
      h_iters.assign(n, (int)t1);
      CU(cudaMemcpyAsync(h_expl.data(), d_expl, sizeof(float) * n, cudaMemcpyDeviceToHost, stream));
    }
    CU(cudaStreamSynchronize(stream));
    CU(cudaEventElapsedTime(&last_solve_ms, ev[2], ev[3]));
    last_setup_ms = 0;
    return check_err();
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// ps_game: a batch of one plus query state
// ---------------------------------------------------------------------------
enum class GState { TreeBuilt = 2, MemoryAllocated = 3, Solved = 4 };

struct ps_game {
  std::unique_ptr<Batch> b;
  Game* g = nullptr;
  GState state = GState::TreeBuilt;
  uint32_t last_iters = 0;
  bool host_dirty = true;
  std::vector<float> hS, hR, hIP, hCH;
  // navigation (query.rs)
  std::vector<size_t> action_history, node_history;
  bool normalized_cached = false;
  uint8_t turn = NOT_DEALT, river = NOT_DEALT;
  int turn_swap = -1, river_swap[2] = {-1, -1}, turn_swapped[2] = {-1, -1};
  int32_t total_bet[2] = {0, 0};
  std::vector<float> weights[2], normalized[2], cfv_cache[2];
  std::vector<std::vector<float>> bcfv_host;  // [ordinal*2+player]
  std::vector<char> bcfv_set;                 // [ordinal*2+player]: values set (from host or device)
  float* fs_block = nullptr;                  // fixed-strategy evaluation vectors (grow-only, freed with the game)
  size_t fs_cap = 0;
  ~ps_game() {
    if (fs_block) {
      if (b && b->stream) cudaStreamSynchronize(b->stream);
      cudaFree(fs_block);
    }
  }
};

namespace {
int sync_host(ps_game* G) {
  if (!G->host_dirty) return PS_OK;
  Game& g = *G->g;
  const SpotDev& s = G->b->h_spots[0];
  G->hS.resize(g.num_storage);
  G->hR.resize(g.num_storage);
  G->hIP.resize(g.num_storage_ip);
  G->hCH.resize(g.num_storage_chance);
  CU(cudaMemcpy(G->hS.data(), s.S, 4 * g.num_storage, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(G->hR.data(), s.R, 4 * g.num_storage, cudaMemcpyDeviceToHost));
  if (g.num_storage_ip) CU(cudaMemcpy(G->hIP.data(), s.ipcfv, 4 * g.num_storage_ip, cudaMemcpyDeviceToHost));
  if (g.num_storage_chance) CU(cudaMemcpy(G->hCH.data(), s.chcfv, 4 * g.num_storage_chance, cudaMemcpyDeviceToHost));
  G->host_dirty = false;
  return PS_OK;
}

int need_ready(ps_game* G) {
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (G->state == GState::Solved) return fail(PS_ERR_STATE, "Game is already solved");
  if (G->state != GState::MemoryAllocated) return fail(PS_ERR_STATE, "Game is not ready");
  return PS_OK;
}

int need_boundaries(ps_game* G) {
  for (int k = 0; k < G->g->num_boundary * 2; ++k)
    if (!G->bcfv_set[k])
      return fail(PS_ERR_STATE, "boundary cfvs empty at ordinal " + std::to_string(k / 2) + ", player " +
                                    std::to_string(k % 2) + " (set_boundary_cfvs not called)");
  return PS_OK;
}

float expl_run(ps_game* G, int* rc) {
  Batch& B = *G->b;
  float e = 0;
  cudaError_t ce = cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream);
  if (ce == cudaSuccess && B.grid_mode)
    ce = B.grid_launch({GRID_EXPL, 0, 0, 0.f, 0, -1, nullptr, nullptr, nullptr});
  else if (ce == cudaSuccess)
    ce = launch_exploitability(B.d_spots, 1, B.d_scratch, B.scratch_floats, B.d_expl, B.d_err, 1, B.block, B.plan,
                               B.stream);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&e, B.d_expl, 4, cudaMemcpyDeviceToHost, B.stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(B.stream);
  if (ce != cudaSuccess) {
    *rc = fail(PS_ERR_CUDA, std::string("exploitability: ") + cudaGetErrorString(ce));
    return 0;
  }
  *rc = B.check_err();
  return e;
}

void assign_zero_weights(ps_game* G) {  // query.rs:886-920
  Game& g = *G->g;
  uint64_t board = 0;
  if (G->turn != NOT_DEALT) board |= 1ull << G->turn;
  if (G->river != NOT_DEALT) board |= 1ull << G->river;
  for (int p = 0; p < 2; ++p) {
    uint64_t dead = (1ull << 52) - 1;
    for (int i = 0; i < g.H[p ^ 1]; ++i) {
      uint64_t m = (1ull << g.cards[p ^ 1][i][0]) | (1ull << g.cards[p ^ 1][i][1]);
      if ((m & board) == 0) dead &= m;
      if (!dead) break;
    }
    dead |= board;
    for (int i = 0; i < g.H[p]; ++i) {
      uint64_t m = (1ull << g.cards[p][i][0]) | (1ull << g.cards[p][i][1]);
      if (m & dead) G->weights[p][i] = 0.f;
    }
  }
}

const ArenaNode& cur(ps_game* G) { return G->g->arena[G->node_history.empty() ? 0 : G->node_history.back()]; }
size_t cur_index(ps_game* G) { return G->node_history.empty() ? 0 : G->node_history.back(); }

bool is_terminal(ps_game* G) {
  const ArenaNode& n = cur(G);
  return n.terminal() || n.amount == G->g->cfg.effective_stack;
}
bool is_chance(ps_game* G) { return cur(G).chance() && !is_terminal(G); }

void apply_swap(ps_game* G, float* v, int p, bool reverse) {  // query.rs:863-883
  Game& g = *G->g;
  int ids[2] = {G->turn_swap >= 0 ? g.iso_perm_turn[G->turn_swap] : -1,
                G->river_swap[0] >= 0 ? g.iso_perm_river[G->river_swap[0]][G->river_swap[1]] : -1};
  if (reverse) std::swap(ids[0], ids[1]);
  for (int id : ids) {
    if (id < 0) continue;
    const auto& perm = g.iso_perm[p][id];
    for (int h = 0; h < g.H[p]; ++h)
      if ((int)perm[h] > h) std::swap(v[h], v[perm[h]]);
  }
}

std::vector<float> normalized_strategy(ps_game* G, const ArenaNode& n) {  // utility.rs:227-250
  Game& g = *G->g;
  int p = n.player, H = g.H[p], hs = g.hs[p], na = n.nch;
  std::vector<float> out((size_t)na * H);
  const float* S = G->hS.data() + n.rs_off;
  float def = 1.0f / (float)na;
  for (int h = 0; h < H; ++h) {
    float d = S[h];
    for (int a = 1; a < na; ++a) d += S[a * hs + h];
    for (int a = 0; a < na; ++a) out[(size_t)a * H + h] = d == 0.0f ? def : S[a * hs + h] / d;
  }
  return out;
}
}  // namespace

extern "C" {

const char* ps_last_error(void) { return g_err.c_str(); }

int ps_hand_table(int32_t* out, int cap) { return build_hand_table(out, cap); }

int ps_parse_bet_sizes(const char* sizes, int is_raise, int32_t* kinds, double* values, int32_t* ints,
                       int32_t* caps, int cap) {
  std::vector<BetSize> v;
  std::string err;
  if (!parse_menu(sizes ? sizes : "", is_raise != 0, v, err)) return fail(PS_ERR_INVALID, err);
  for (size_t k = 0; k < v.size() && (int)k < cap; ++k) {
    kinds[k] = (int32_t)v[k].kind;
    values[k] = v[k].ratio;
    ints[k] = v[k].n;
    caps[k] = v[k].cap;
  }
  return (int)v.size();
}

int ps_discount_params(uint32_t t, float out[3]) {
  Discount d = discount_params(t);
  out[0] = d.alpha;
  out[1] = d.beta;
  out[2] = d.gamma;
  return PS_OK;
}

int ps_game_new(const ps_card_config* cc, const ps_tree_config* tc, ps_game** out) {
  if (!cc || !tc || !out || !cc->range[0] || !cc->range[1]) return fail(PS_ERR_INVALID, "null argument");
  *out = nullptr;
  TreeCfg t;
  std::string err;
  if (!parse_tree_config(tc, t, err)) return fail(PS_ERR_INVALID, err);
  auto g = std::make_unique<Game>();
  uint8_t board[5] = {cc->flop[0], cc->flop[1], cc->flop[2], cc->turn, cc->river};
  if (!g->init(cc->range[0], cc->range[1], board, t, err)) return fail(PS_ERR_INVALID, err);
  auto* G = new ps_game();
  G->b = std::make_unique<Batch>();
  G->g = g.get();
  G->b->games.push_back(std::move(g));
  G->bcfv_host.assign((size_t)G->g->num_boundary * 2, {});
  G->bcfv_set.assign((size_t)G->g->num_boundary * 2, 0);
  for (int p = 0; p < 2; ++p) {
    G->weights[p].assign(G->g->H[p], 0.f);
    G->normalized[p].assign(G->g->H[p], 0.f);
    G->cfv_cache[p].assign(G->g->H[p], 0.f);
  }
  *out = G;
  return PS_OK;
}

void ps_game_free(ps_game* G) { delete G; }

int ps_game_memory_usage(ps_game* G, uint64_t* bytes) {
  if (!G || !bytes) return fail(PS_ERR_INVALID, "null argument");
  Game& g = *G->g;
  *bytes = 4 * (2 * g.num_storage + g.num_storage_ip + g.num_storage_chance);
  return PS_OK;
}

int ps_game_set_terminals_first(ps_game* G, int enable) {
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (G->state != GState::TreeBuilt) return fail(PS_ERR_STATE, "choose the program before allocate_memory");
  std::string err;
  if (!G->g->recompile(enable != 0, err)) return fail(PS_ERR_INVALID, err);
  G->g->program_choice = enable != 0;
  return PS_OK;
}

int ps_game_program_info(ps_game* G, int64_t out[12]) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  const Game& g = *G->g;
  out[0] = g.num_slots;
  out[1] = g.vstride;
  int64_t S = 0;
  for (const auto& n : g.arena)
    if (!n.terminal() && !n.chance()) S += (int64_t)n.nch * g.H[n.player];
  for (int p = 0; p < 2; ++p) {
    const Program& P = g.prog[p];
    int64_t ne = 0, nt = 0, ng = 0;
    for (const auto& st : P.steps) {
      ne += st.n_elem;
      nt += st.n_term;
      ng += st.n_groups;
    }
    out[2 + p] = (int64_t)P.steps.size();
    out[4 + p] = ne;
    out[6 + p] = nt;
    out[8 + p] = ng;
  }
  out[10] = S;
  out[11] = (int64_t)g.boards.size();
  return PS_OK;
}

int ps_game_allocate_memory(ps_game* G, int enable_compression) {
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (enable_compression) return fail(PS_ERR_UNSUPPORTED, "compressed (16-bit) storage is not supported: state is FP32");
  if (G->state != GState::TreeBuilt) return PS_OK;
  // one game on one CTA is latency-bound: its board tables go to shared
  // memory when it has a single board, and every warp holds a terminal scan
  // buffer (occupancy does not matter for a lone CTA)
  ps_batch_opts o{};
  o.block_threads = 0;
  o.sort_by_cost = 1;
  o.stage_tables = PS_SINGLE_STAGE;
  o.scan_buffers = PS_SINGLE_BUFS;
  int rc = G->b->build(&o);
  if (!rc) rc = G->b->run_setup();
  if (rc) return rc;
  G->state = GState::MemoryAllocated;
  ps_back_to_root(G);
  return PS_OK;
}

int ps_solve(ps_game* G, uint32_t max_iter, float target, int print, float* out) {
  int rc = need_ready(G);
  if (rc) return rc;
  if ((rc = need_boundaries(G))) return rc;
  rc = G->b->solve(max_iter, &target, false);
  if (rc) return rc;
  float e = G->b->h_expl[0];
  G->last_iters = (uint32_t)G->b->h_iters[0];
  if (print) printf("iteration: %u / %u (exploitability = %.4e)\n", G->last_iters, max_iter, e);
  G->host_dirty = true;
  if ((rc = ps_finalize(G))) return rc;
  if (out) *out = e;
  return PS_OK;
}

int ps_last_iterations(ps_game* G, uint32_t* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  *out = G->last_iters;
  return PS_OK;
}

int ps_solve_step(ps_game* G, uint32_t t) {
  int rc = need_ready(G);
  if (rc) return rc;
  if ((rc = need_boundaries(G))) return rc;
  Batch& B = *G->b;
  if ((rc = B.ensure_disc(t + 1))) return rc;
  CU(cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream));
  if (B.grid_mode)
    CU(B.grid_launch({GRID_ITERATE, (int)t, (int)t + 1, 0.f, 0, -1, nullptr, nullptr, nullptr}));
  else
    CU(launch_iterate(B.d_spots, 1, B.d_disc, (int)t, (int)t + 1, B.d_scratch, B.scratch_floats, B.d_err, 1,
                      B.block, B.plan, B.stream));
  G->host_dirty = true;
  return B.check_err();
}

int ps_compute_exploitability(ps_game* G, float* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Game is not ready");
  int rc = need_boundaries(G);
  if (rc) return rc;
  float e = expl_run(G, &rc);
  if (rc) return rc;
  *out = e;
  return PS_OK;
}

int ps_compute_exploitability_noalloc(ps_game* G, float* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Game is not ready");
  int rc = need_boundaries(G);
  if (rc) return rc;
  const size_t need = (size_t)G->g->num_slots * G->g->vstride;
  if (need > kFixedScratchFloats)
    return fail(PS_ERR_INVALID, "game needs " + std::to_string(need) + " floats of working slots; the fixed array of "
                                    "the no-allocation path holds " + std::to_string(kFixedScratchFloats));
  Batch& B = *G->b;
  float e = 0;
  int err = 0;
  CU(launch_exploitability_fixed(B.d_spots, need, B.block, B.plan, B.stream, &e, &err));
  if (err) return fail(PS_ERR_DEVICE, "kernel error flag " + std::to_string(err));
  *out = e;
  return PS_OK;
}

int ps_finalize(ps_game* G) {
  int rc = need_ready(G);
  if (rc) return rc;
  if ((rc = need_boundaries(G))) return rc;
  Batch& B = *G->b;
  CU(cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream));
  CU(B.average(1, 0, nullptr, nullptr, -1, nullptr));
  if ((rc = B.check_err())) return rc;
  G->state = GState::Solved;
  G->host_dirty = true;
  if ((rc = sync_host(G))) return rc;
  auto h = G->action_history;  // set_solved re-applies the history (interpreter.rs:67-71)
  ps_back_to_root(G);
  for (size_t a : h) ps_play(G, (int64_t)a);
  return PS_OK;
}

int ps_root_cfvalues_with_reach(ps_game* G, int player, const float* opp_reach, float* out) {
  if (!G || !out || (player != 0 && player != 1)) return fail(PS_ERR_INVALID, "bad argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Game is not ready");
  int rc = need_boundaries(G);
  if (rc) return rc;
  Batch& B = *G->b;
  Game& g = *G->g;
  const int o = player ^ 1;
  float* d_reach = nullptr;
  float* d_out = nullptr;
  std::vector<float> r(g.hs[o], 0.f);
  for (int h = 0; h < g.H[o]; ++h) r[h] = opp_reach ? opp_reach[h] : g.w[o][h];
  // freed on every return (cudaFree waits for the device, so an error path
  // never frees a buffer that queued work still reads)
  CU(cudaMalloc(&d_reach, 4 * r.size()));
  std::unique_ptr<float, decltype(&cudaFree)> k1(d_reach, &cudaFree);
  CU(cudaMalloc(&d_out, 4 * (size_t)g.hs[player]));
  std::unique_ptr<float, decltype(&cudaFree)> k2(d_out, &cudaFree);
  CU(cudaMemcpyAsync(d_reach, r.data(), 4 * r.size(), cudaMemcpyHostToDevice, B.stream));
  CU(cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream));
  CU(B.average(0, player, d_reach, d_out, -1, nullptr));
  CU(cudaMemcpyAsync(out, d_out, 4 * (size_t)g.H[player], cudaMemcpyDeviceToHost, B.stream));
  CU(cudaStreamSynchronize(B.stream));
  return B.check_err();
}

// Fixed-strategy evaluation and its adjoint (no reference counterpart: the
// reference has no gradients).  Both passes use the average strategy, the
// boundary values as set, and the given initial weights instead of the game's.
static int fixed_strategy_run(ps_game* G, const float* w0, const float* w1, const float* g0, const float* g1,
                              float* cfv0, float* cfv1, float* dw0, float* dw1, float* dbcfv, bool on_device) {
  if (!G || !w0 || !w1) return fail(PS_ERR_INVALID, "null argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Game is not ready");
  int rc = need_boundaries(G);
  if (rc) return rc;
  Batch& B = *G->b;
  Game& g = *G->g;
  if (!g.iso_list.empty())
    return fail(PS_ERR_UNSUPPORTED, "fixed-strategy evaluation with arbitrary weights needs a game without "
                                    "isomorphic chance pruning (its suit swaps assume the game's own ranges)");
  const bool adjoint = dw0 || dw1 || dbcfv;
  const size_t hs0 = g.hs[0], hs1 = g.hs[1], nb = (size_t)g.num_boundary;
  const size_t H0 = g.H[0], H1 = g.H[1];
  // one device block, kept by the game: w0 w1 c0 c1 (g0 g1 a0 a1 when adjoint) then the boundary gradients
  const size_t nvec = adjoint ? 8 : 4;
  const size_t vec = std::max(hs0, hs1);
  const size_t nbg = adjoint ? nb * 2 * (size_t)g.vstride : 0;
  const size_t need = 4 * (nvec * vec + nbg + 4);
  if (G->fs_cap < need) {
    cudaFree(G->fs_block);
    G->fs_block = nullptr;
    G->fs_cap = 0;
    CU(cudaMalloc(&G->fs_block, need));
    G->fs_cap = need;
  }
  float* d = G->fs_block;
  float* dv[8];
  for (size_t k = 0; k < nvec; ++k) dv[k] = d + k * vec;
  float* d_bg = nbg ? d + nvec * vec : nullptr;
  const cudaMemcpyKind in = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind out = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  CU(cudaMemsetAsync(d, 0, 4 * (nvec * vec + nbg), B.stream));
  CU(cudaMemcpyAsync(dv[0], w0, 4 * H0, in, B.stream));
  CU(cudaMemcpyAsync(dv[1], w1, 4 * H1, in, B.stream));
  if (adjoint) {
    if (g0) CU(cudaMemcpyAsync(dv[4], g0, 4 * H0, in, B.stream));
    if (g1) CU(cudaMemcpyAsync(dv[5], g1, 4 * H1, in, B.stream));
  }
  CU(cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream));
  // forward: cfv_p from the opponent's weights (utility.rs:422-443)
  CU(B.average(0, 0, dv[1], dv[2], -1, d_bg));
  CU(B.average(0, 1, dv[0], dv[3], -1, d_bg));
  if (adjoint) {
    // cotangent of cfv_0 flows into player 1's weights and player 0's boundary values, and vice versa
    CU(B.average(0, 1, dv[4], dv[7], 0, d_bg));
    CU(B.average(0, 0, dv[5], dv[6], 1, d_bg));
  }
  if (cfv0) CU(cudaMemcpyAsync(cfv0, dv[2], 4 * H0, out, B.stream));
  if (cfv1) CU(cudaMemcpyAsync(cfv1, dv[3], 4 * H1, out, B.stream));
  if (dw0) CU(cudaMemcpyAsync(dw0, dv[6], 4 * H0, out, B.stream));
  if (dw1) CU(cudaMemcpyAsync(dw1, dv[7], 4 * H1, out, B.stream));
  if (dbcfv && nb) {  // [nb][2][vstride] -> [nb][H0 + H1], one strided copy per player
    CU(cudaMemcpy2DAsync(dbcfv, (H0 + H1) * 4, d_bg, 2 * g.vstride * 4, H0 * 4, nb, out, B.stream));
    CU(cudaMemcpy2DAsync(dbcfv + H0, (H0 + H1) * 4, d_bg + g.vstride, 2 * g.vstride * 4, H1 * 4, nb, out, B.stream));
  }
  CU(cudaStreamSynchronize(B.stream));
  return B.check_err();
}

int ps_boundary_reach(ps_game* G, float* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Game is not ready");
  int rc = need_boundaries(G);
  if (rc) return rc;
  Batch& B = *G->b;
  Game& g = *G->g;
  const size_t nb = (size_t)g.num_boundary;
  if (nb == 0) return PS_OK;
  const size_t vec = std::max(g.hs[0], g.hs[1]);
  float* d = nullptr;
  CU(cudaMalloc(&d, 4 * (nb * 2 * (size_t)g.vstride + vec)));
  std::unique_ptr<float, decltype(&cudaFree)> keep(d, &cudaFree);
  float* d_root = d + nb * 2 * (size_t)g.vstride;
  CU(cudaMemsetAsync(d, 0, 4 * nb * 2 * (size_t)g.vstride, B.stream));
  CU(cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream));
  // traverser 0 records player 1's reach at every boundary, traverser 1 player 0's
  for (int p = 0; p < 2; ++p) CU(B.average(0, p, nullptr, d_root, -1, nullptr, d));
  for (size_t k = 0; k < nb; ++k)
    for (int p = 0; p < 2; ++p)
      CU(cudaMemcpyAsync(out + k * (g.H[0] + g.H[1]) + (p ? g.H[0] : 0), d + (k * 2 + p) * g.vstride,
                         4 * (size_t)g.H[p], cudaMemcpyDeviceToHost, B.stream));
  CU(cudaStreamSynchronize(B.stream));
  return B.check_err();
}

int ps_boundary_river_reduce(int32_t n, const uint8_t* boards, const float* pots, const float* stacks,
                             const void* net, int32_t net_bf16, const float* reach, const int32_t* hands, int32_t H,
                             float* out, void* stream) {
  if (n < 0 || H < 0 || H > 1326 || (n > 0 && (!boards || !pots || !stacks || !net || !reach || !hands || !out)))
    return fail(PS_ERR_INVALID, "bad argument");
  if (n == 0 || H == 0) return PS_OK;
  std::vector<uint8_t> hb((size_t)n * 4);
  std::vector<float> dn(n);
  for (int i = 0; i < n; ++i) {
    uint64_t seen = 0;
    for (int k = 0; k < 4; ++k) {
      const uint8_t c = boards[4 * i + k];
      if (c >= 52 || (seen >> c & 1)) return fail(PS_ERR_INVALID, "boards must hold 4 distinct cards below 52");
      seen |= 1ull << c;
      hb[4 * i + k] = c;
    }
    dn[i] = (float)((double)pots[i] + (double)stacks[i]);
  }
  cudaStream_t s = (cudaStream_t)stream;
  StagingLease lease;
  CU(lease.acquire(hb.size() + 4 * dn.size() + 16));
  lease.using_stream(s);
  char* d = lease.ptr;
  float* d_dn = (float*)(d + ((hb.size() + 15) & ~(size_t)15));
  CU(cudaMemcpyAsync(d, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d_dn, dn.data(), 4 * dn.size(), cudaMemcpyHostToDevice, s));
  CU(launch_boundary_river_reduce(n, (const uint8_t*)d, d_dn, net, net_bf16 ? 1 : 0, reach, hands, H, out, s));
  CU(cudaStreamSynchronize(s));
  lease.done();
  return PS_OK;
}

int ps_boundary_first_layer(int32_t n, const uint8_t* boards, const float* pots, const float* stacks,
                            const float* base, const float* percard, const float* wcols, const float* bias, int32_t h,
                            void* out, int32_t out_bf16, void* stream) {
  if (n < 0 || h < 0 || (n > 0 && h > 0 && (!boards || !pots || !stacks || !base || !percard || !wcols || !out)))
    return fail(PS_ERR_INVALID, "bad argument");
  if (n == 0 || h == 0) return PS_OK;
  if (h > kMaxFirstLayerWidth) return fail(PS_ERR_INVALID, "first layer wider than 8192");
  std::vector<uint8_t> hb((size_t)n * 4);
  for (int i = 0; i < n; ++i) {
    uint64_t seen = 0;
    for (int k = 0; k < 4; ++k) {
      const uint8_t c = boards[4 * i + k];
      if (c >= 52 || (seen >> c & 1)) return fail(PS_ERR_INVALID, "boards must hold 4 distinct cards below 52");
      seen |= 1ull << c;
      hb[4 * i + k] = c;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  const size_t ob = (hb.size() + 15) & ~(size_t)15;
  StagingLease lease;
  CU(lease.acquire(ob + 8 * (size_t)n + 16));
  lease.using_stream(s);
  char* d = lease.ptr;
  float* d_pot = (float*)(d + ob);
  float* d_stack = d_pot + n;
  CU(cudaMemcpyAsync(d, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d_pot, pots, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d_stack, stacks, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
  CU(launch_boundary_first_layer(n, (const uint8_t*)d, d_pot, d_stack, base, percard, wcols, bias, h, out,
                                 out_bf16 ? 1 : 0, s));
  CU(cudaStreamSynchronize(s));
  lease.done();
  return PS_OK;
}

int ps_eval_fixed_strategy(ps_game* G, const float* w0, const float* w1, float* cfv0, float* cfv1) {
  return fixed_strategy_run(G, w0, w1, nullptr, nullptr, cfv0, cfv1, nullptr, nullptr, nullptr, false);
}

int ps_eval_fixed_strategy_adjoint(ps_game* G, const float* w0, const float* w1, const float* g0, const float* g1,
                                   float* dw0, float* dw1, float* dbcfv) {
  if (!dw0 || !dw1) return fail(PS_ERR_INVALID, "null argument");
  return fixed_strategy_run(G, w0, w1, g0, g1, nullptr, nullptr, dw0, dw1, dbcfv, false);
}

int ps_eval_fixed_strategy_ex(ps_game* G, const float* w0, const float* w1, float* cfv0, float* cfv1,
                              int32_t on_device) {
  return fixed_strategy_run(G, w0, w1, nullptr, nullptr, cfv0, cfv1, nullptr, nullptr, nullptr, on_device != 0);
}

int ps_eval_fixed_strategy_adjoint_ex(ps_game* G, const float* w0, const float* w1, const float* g0,
                                      const float* g1, float* dw0, float* dw1, float* dbcfv, int32_t on_device) {
  if (!dw0 || !dw1) return fail(PS_ERR_INVALID, "null argument");
  return fixed_strategy_run(G, w0, w1, g0, g1, nullptr, nullptr, dw0, dw1, dbcfv, on_device != 0);
}

int ps_num_private_hands(ps_game* G, int p) { return G ? G->g->H[p & 1] : fail(PS_ERR_INVALID, "null game"); }

int ps_private_cards(ps_game* G, int p, uint8_t* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  for (int h = 0; h < G->g->H[p & 1]; ++h) {
    out[2 * h] = G->g->cards[p & 1][h][0];
    out[2 * h + 1] = G->g->cards[p & 1][h][1];
  }
  return PS_OK;
}

int ps_initial_weights(ps_game* G, int p, float* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  std::copy(G->g->w[p & 1].begin(), G->g->w[p & 1].end(), out);
  return PS_OK;
}

double ps_num_combinations(ps_game* G) { return G ? G->g->num_combinations : 0.0; }
int64_t ps_num_nodes(ps_game* G) { return G ? (int64_t)G->g->arena.size() : -1; }

int ps_node_info(ps_game* G, int64_t idx, int32_t out[8]) {
  if (!G || idx < 0 || idx >= (int64_t)G->g->arena.size()) return fail(PS_ERR_INVALID, "bad node index");
  const ArenaNode& n = G->g->arena[idx];
  out[0] = n.player;
  out[1] = n.amount;
  out[2] = n.turn;
  out[3] = n.river;
  out[4] = n.nch;
  out[5] = (int32_t)n.child_off;
  out[6] = n.prev.kind;
  out[7] = n.prev.amount;
  return PS_OK;
}

int ps_child_indices(ps_game* G, int64_t idx, int64_t* out, int cap) {
  if (!G || idx < 0 || idx >= (int64_t)G->g->arena.size()) return fail(PS_ERR_INVALID, "bad node index");
  const ArenaNode& n = G->g->arena[idx];
  if (n.terminal()) return 0;
  for (int c = 0; c < n.nch && c < cap; ++c) out[c] = idx + n.child_off + c;
  return n.nch;
}

int ps_strategy_at_index(ps_game* G, int64_t idx, float* out) {
  if (!G || idx < 0 || idx >= (int64_t)G->g->arena.size()) return fail(PS_ERR_INVALID, "bad node index");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  const ArenaNode& n = G->g->arena[idx];
  if (n.terminal() || n.chance()) return fail(PS_ERR_INVALID, "strategy_at_index requires a decision node");
  int rc = sync_host(G);
  if (rc) return rc;
  auto v = normalized_strategy(G, n);
  std::copy(v.begin(), v.end(), out);
  return (int)v.size();
}

int64_t ps_node_storage(ps_game* G, int64_t idx, int which, float* out) {
  if (!G || idx < 0 || idx >= (int64_t)G->g->arena.size()) return fail(PS_ERR_INVALID, "bad node index");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  int rc = sync_host(G);
  if (rc) return rc;
  Game& g = *G->g;
  const ArenaNode& n = g.arena[idx];
  if (n.terminal()) return 0;
  if (which == 4) {
    if (!n.chance() || n.ch_off == 0xFFFFFFFFu) return 0;
    int sp = (n.player & PL_MASK) ^ 1;
    std::copy(G->hCH.begin() + n.ch_off, G->hCH.begin() + n.ch_off + g.H[sp], out);
    return g.H[sp];
  }
  if (n.chance()) return 0;
  if (which == 3) {
    if (n.ip_off == 0xFFFFFFFFu) return 0;
    std::copy(G->hIP.begin() + n.ip_off, G->hIP.begin() + n.ip_off + g.H[1], out);
    return g.H[1];
  }
  const auto& src = which == 1 ? G->hS : G->hR;
  int p = n.player, H = g.H[p], hs = g.hs[p];
  for (int a = 0; a < n.nch; ++a)
    for (int h = 0; h < H; ++h) out[(size_t)a * H + h] = src[n.rs_off + (size_t)a * hs + h];
  return (int64_t)n.nch * H;
}

int ps_seed_node_storage(ps_game* G, int64_t idx, int which, const float* v, int64_t n) {
  if (!G || !v || idx < 0 || idx >= (int64_t)G->g->arena.size() || (which != 1 && which != 2))
    return fail(PS_ERR_INVALID, "bad argument");
  if (G->state != GState::MemoryAllocated) return fail(PS_ERR_STATE, "Game is not ready");
  Game& g = *G->g;
  const ArenaNode& nd = g.arena[idx];
  if (nd.terminal() || nd.chance()) return fail(PS_ERR_INVALID, "seed requires a decision node");
  int p = nd.player, H = g.H[p], hs = g.hs[p];
  if (n != (int64_t)nd.nch * H) return fail(PS_ERR_INVALID, "expected num_actions * num_hands values");
  std::vector<float> rows((size_t)nd.nch * hs, 0.f);
  for (int a = 0; a < nd.nch; ++a)
    for (int h = 0; h < H; ++h) rows[(size_t)a * hs + h] = v[(size_t)a * H + h];
  const SpotDev& s = G->b->h_spots[0];
  float* dst = (which == 1 ? s.S : s.R) + nd.rs_off;
  CU(cudaMemcpy(dst, rows.data(), 4 * rows.size(), cudaMemcpyHostToDevice));
  G->host_dirty = true;
  return PS_OK;
}

int ps_same_hand_index(ps_game* G, int p, uint16_t* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  std::copy(G->g->same[p & 1].begin(), G->g->same[p & 1].end(), out);
  return PS_OK;
}

static int find_board(ps_game* G, int turn, int river) {
  Game& g = *G->g;
  for (size_t b = 0; b < g.boards.size(); ++b)
    if (g.boards[b][3] == (uint8_t)turn && g.boards[b][4] == (uint8_t)river) return (int)b;
  return -1;
}

int ps_hand_strength(ps_game* G, int turn, int river, int p, uint16_t* strength, uint16_t* index) {
  if (!G || G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  int b = find_board(G, turn, river);
  if (b < 0) return fail(PS_ERR_INVALID, "board not in this game");
  Game& g = *G->g;
  const SpotDev& s = G->b->h_spots[0];
  int V = 0;
  CU(cudaMemcpy(&V, s.nvalid[p] + b, 4, cudaMemcpyDeviceToHost));
  std::vector<uint16_t> ord(V), thr((size_t)g.hs[p] * kThrWords);
  CU(cudaMemcpy(ord.data(), s.gidx[p] + (size_t)b * 3 * g.hs[p], 2 * (size_t)V, cudaMemcpyDeviceToHost));
  // the strength of each ordered hand: recover from the opponent's thresholds is
  // indirect, so evaluate it on the host with the shared evaluator
  std::vector<int32_t> table(kHandTableSize);
  build_hand_table(table.data(), kHandTableSize);
  strength[0] = 0;
  index[0] = 0;
  for (int k = 0; k < V; ++k) {
    int h = ord[k];
    uint16_t st = 0;
    if (g.boards[b][4] != NOT_DEALT) {
      int c7[7] = {g.boards[b][0], g.boards[b][1], g.boards[b][2], g.boards[b][3], g.boards[b][4],
                   g.cards[p][h][0], g.cards[p][h][1]};
      st = (uint16_t)(table_index(table.data(), kHandTableSize, hand_value7(c7)) + 1);
    }
    strength[k + 1] = st;
    index[k + 1] = (uint16_t)h;
  }
  strength[V + 1] = 0xFFFF;
  index[V + 1] = 0xFFFF;
  return V + 2;
}

int ps_valid_indices(ps_game* G, int turn, int river, int p, uint16_t* out) {
  if (!G || G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  int b = find_board(G, turn, river);
  if (b < 0) return fail(PS_ERR_INVALID, "board not in this game");
  Game& g = *G->g;
  const SpotDev& s = G->b->h_spots[0];
  std::vector<uint16_t> thr((size_t)g.hs[p] * kThrWords);
  CU(cudaMemcpy(thr.data(), s.thr[p] + (size_t)b * g.hs[p] * kThrWords, 2 * thr.size(), cudaMemcpyDeviceToHost));
  int n = 0;
  for (int h = 0; h < g.H[p]; ++h)
    if (thr[(size_t)h * kThrWords] != 0xFFFF || thr[(size_t)h * kThrWords + 1] != 0xFFFF) out[n++] = (uint16_t)h;
  return n;
}

int64_t ps_num_boundary_nodes(ps_game* G) { return G ? G->g->num_boundary : -1; }

int ps_boundary_node_indices(ps_game* G, int64_t* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  for (size_t i = 0; i < G->g->bnd_ordinal.size(); ++i)
    if (G->g->bnd_ordinal[i] >= 0) out[G->g->bnd_ordinal[i]] = (int64_t)i;
  return PS_OK;
}

int ps_set_boundary_cfvs(ps_game* G, int64_t ordinal, int p, const float* cfvs, int64_t n) {
  if (!G || !cfvs || (p != 0 && p != 1)) return fail(PS_ERR_INVALID, "bad argument");
  Game& g = *G->g;
  if (ordinal < 0 || ordinal >= g.num_boundary) return PS_OK;  // ignored like the reference (interpreter.rs:343-348)
  if (n != g.H[p]) return fail(PS_ERR_INVALID, "cfvs must have one value per private hand");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "allocate memory before setting boundary values");
  G->bcfv_host[ordinal * 2 + p].assign(cfvs, cfvs + n);
  const SpotDev& s = G->b->h_spots[0];
  CU(cudaMemcpy((float*)s.bcfv + ((size_t)ordinal * 2 + p) * g.vstride, cfvs, 4 * (size_t)n, cudaMemcpyHostToDevice));
  G->bcfv_set[ordinal * 2 + p] = 1;
  return PS_OK;
}

int ps_set_boundary_cfvs_all(ps_game* G, const float* values, int32_t on_device) {
  if (!G || (!values && G && G->g->num_boundary > 0)) return fail(PS_ERR_INVALID, "bad argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "allocate memory before setting boundary values");
  Game& g = *G->g;
  const size_t nb = (size_t)g.num_boundary, H0 = g.H[0], H1 = g.H[1];
  if (nb == 0) return PS_OK;
  Batch& B = *G->b;
  const SpotDev& s = B.h_spots[0];
  // [nb][H0 + H1] rows -> the device layout [nb][2][vstride], one strided copy per player
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CU(cudaMemcpy2DAsync((float*)s.bcfv, 2 * g.vstride * 4, values, (H0 + H1) * 4, H0 * 4, nb, kind, B.stream));
  CU(cudaMemcpy2DAsync((float*)s.bcfv + g.vstride, 2 * g.vstride * 4, values + H0, (H0 + H1) * 4, H1 * 4, nb, kind,
                       B.stream));
  CU(cudaStreamSynchronize(B.stream));
  for (size_t k = 0; k < nb; ++k) {
    if (!on_device) {
      G->bcfv_host[k * 2].assign(values + k * (H0 + H1), values + k * (H0 + H1) + H0);
      G->bcfv_host[k * 2 + 1].assign(values + k * (H0 + H1) + H0, values + (k + 1) * (H0 + H1));
    }
    G->bcfv_set[k * 2] = G->bcfv_set[k * 2 + 1] = 1;
  }
  return PS_OK;
}

// ---- navigation (query.rs) ----
int ps_back_to_root(ps_game* G) {
  if (!G) return fail(PS_ERR_INVALID, "null game");
  Game& g = *G->g;
  G->action_history.clear();
  G->node_history.clear();
  G->normalized_cached = false;
  G->turn = g.turn;
  G->river = g.river;
  G->turn_swap = -1;
  G->river_swap[0] = G->river_swap[1] = -1;
  G->turn_swapped[0] = G->turn_swapped[1] = -1;
  G->total_bet[0] = G->total_bet[1] = 0;
  for (int p = 0; p < 2; ++p) G->weights[p] = g.w[p];
  assign_zero_weights(G);
  return PS_OK;
}

int ps_is_terminal_node(ps_game* G) { return G ? (int)is_terminal(G) : fail(PS_ERR_INVALID, "null game"); }
int ps_is_chance_node(ps_game* G) { return G ? (int)is_chance(G) : fail(PS_ERR_INVALID, "null game"); }
int ps_current_player(ps_game* G) { return G ? (int)cur(G).player : fail(PS_ERR_INVALID, "null game"); }
int64_t ps_current_node_index(ps_game* G) { return G ? (int64_t)cur_index(G) : -1; }

int ps_available_actions(ps_game* G, int32_t* kinds, int32_t* amounts, int cap) {
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (is_terminal(G)) return 0;
  const ArenaNode& n = cur(G);
  size_t idx = cur_index(G);
  for (int c = 0; c < n.nch && c < cap; ++c) {
    const ArenaNode& ch = G->g->arena[idx + n.child_off + c];
    kinds[c] = ch.prev.kind;
    amounts[c] = ch.prev.amount;
  }
  return n.nch;
}

uint64_t ps_possible_cards(ps_game* G) {  // query.rs:100-136
  if (!G || !is_chance(G)) return 0;
  Game& g = *G->g;
  uint64_t board = (1ull << g.flop[0]) | (1ull << g.flop[1]) | (1ull << g.flop[2]);
  if (G->turn != NOT_DEALT) board |= 1ull << G->turn;
  uint64_t dead = 0;
  for (int card = 0; card < 52; ++card) {
    uint64_t nb = board | (1ull << card);
    bool alive = false;
    if (nb != board) {
      for (int i = 0; i < g.H[0] && !alive; ++i) {
        uint64_t om = (1ull << g.cards[0][i][0]) | (1ull << g.cards[0][i][1]);
        if (om & nb) continue;
        uint64_t cm = om | nb;
        for (int j = 0; j < g.H[1]; ++j) {
          uint64_t im = (1ull << g.cards[1][j][0]) | (1ull << g.cards[1][j][1]);
          if (!(im & cm)) {
            alive = true;
            break;
          }
        }
      }
    }
    if (!alive) dead |= 1ull << card;
  }
  return ((1ull << 52) - 1) ^ dead;
}

int ps_strategy(ps_game* G, float* out) {  // query.rs:346-378
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  if (is_terminal(G)) return fail(PS_ERR_STATE, "Terminal node is not allowed");
  if (is_chance(G)) return fail(PS_ERR_STATE, "Chance node is not allowed");
  int rc = sync_host(G);
  if (rc) return rc;
  const ArenaNode& n = cur(G);
  auto v = normalized_strategy(G, n);
  int H = G->g->H[n.player];
  for (int a = 0; a < n.nch; ++a) apply_swap(G, v.data() + (size_t)a * H, n.player, false);
  std::copy(v.begin(), v.end(), out);
  return (int)v.size();
}

int ps_play(ps_game* G, int64_t action) {  // query.rs:186-335
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  if (is_terminal(G)) return fail(PS_ERR_STATE, "Terminal node is not allowed");
  Game& g = *G->g;
  size_t idx = cur_index(G);
  const ArenaNode& n = g.arena[idx];
  if (is_chance(G)) {
    bool is_turn = G->turn == NOT_DEALT;
    int actual = action < 0 ? __builtin_ctzll(ps_possible_cards(G)) : (int)action;
    int card = actual;
    if (G->turn_swapped[0] >= 0) {
      int s1 = G->turn_swapped[0], s2 = G->turn_swapped[1];
      if ((actual & 3) == s1) card = actual - s1 + s2;
      else if ((actual & 3) == s2) card = actual + s1 - s2;
    }
    int ai = -1;
    for (int c = 0; c < n.nch; ++c)
      if (g.arena[idx + n.child_off + c].prev.amount == card) {
        ai = c;
        break;
      }
    if (ai < 0) {
      const auto& iref = n.turn == NOT_DEALT ? g.iso_ref_turn : g.iso_ref_river[n.turn];
      const auto& icard = n.turn == NOT_DEALT ? g.iso_card_turn : g.iso_card_river[n.turn & 3];
      for (size_t i = 0; i < iref.size(); ++i)
        if (card == icard[i]) {
          ai = iref[i];
          if (is_turn) {
            G->turn_swapped[0] = card & 3;
            G->turn_swapped[1] = g.arena[idx + n.child_off + ai].prev.amount & 3;
            G->turn_swap = card & 3;
          } else {
            G->river_swap[0] = G->turn & 3;
            G->river_swap[1] = icard[i] & 3;
          }
          break;
        }
    }
    if (ai < 0) return fail(PS_ERR_INVALID, "Invalid action");
    G->node_history.push_back(idx + n.child_off + ai);
    if (is_turn) G->turn = (uint8_t)actual;
    else G->river = (uint8_t)actual;
    assign_zero_weights(G);
  } else {
    if (action < 0 || action >= n.nch) return fail(PS_ERR_INVALID, "Invalid action");
    int rc = sync_host(G);
    if (rc) return rc;
    int p = n.player, H = g.H[p];
    if (n.nch > 1) {
      std::vector<float> st((size_t)n.nch * H);
      rc = ps_strategy(G, st.data());
      if (rc < 0) return rc;
      for (int h = 0; h < H; ++h) G->weights[p][h] *= st[(size_t)action * H + h];
    }
    for (int h = 0; h < H; ++h) G->cfv_cache[p][h] = G->hR[n.rs_off + (size_t)action * g.hs[p] + h];
    const Act& pa = g.arena[idx + n.child_off + action].prev;
    if (pa.kind == ACT_CALL) {
      G->total_bet[p] = G->total_bet[p ^ 1];
    } else if (pa.kind == ACT_BET || pa.kind == ACT_RAISE || pa.kind == ACT_ALLIN) {
      int prev = (n.prev.kind == ACT_BET || n.prev.kind == ACT_RAISE || n.prev.kind == ACT_ALLIN) ? n.prev.amount : 0;
      int to_call = G->total_bet[p ^ 1] - G->total_bet[p];
      G->total_bet[p] += pa.amount - prev + to_call;
    }
    G->node_history.push_back(idx + n.child_off + action);
  }
  G->action_history.push_back((size_t)action);
  G->normalized_cached = false;
  return PS_OK;
}

int ps_cache_normalized_weights(ps_game* G) {  // query.rs:498-567
  if (!G) return fail(PS_ERR_INVALID, "null game");
  if (G->normalized_cached) return PS_OK;
  Game& g = *G->g;
  uint64_t board = 0;
  if (G->turn != NOT_DEALT) board |= 1ull << G->turn;
  if (G->river != NOT_DEALT) board |= 1ull << G->river;
  double ws[2] = {0, 0}, wm[2][52];
  for (int p = 0; p < 2; ++p) {
    for (int c = 0; c < 52; ++c) wm[p][c] = 0;
    for (int i = 0; i < g.H[p]; ++i) {
      int c1 = g.cards[p][i][0], c2 = g.cards[p][i][1];
      if (((1ull << c1) | (1ull << c2)) & board) continue;
      double w = G->weights[p][i];
      ws[p] += w;
      wm[p][c1] += w;
      wm[p][c2] += w;
    }
  }
  for (int p = 0; p < 2; ++p)
    for (int i = 0; i < g.H[p]; ++i) {
      int c1 = g.cards[p][i][0], c2 = g.cards[p][i][1];
      if (((1ull << c1) | (1ull << c2)) & board) {
        G->normalized[p][i] = 0.f;
        continue;
      }
      uint16_t si = g.same[p][i];
      double osame = si == 0xFFFF ? 0.0 : (double)G->weights[p ^ 1][si];
      double ow = ws[p ^ 1] + osame - wm[p ^ 1][c1] - wm[p ^ 1][c2];
      G->normalized[p][i] = G->weights[p][i] * (float)ow;
    }
  G->normalized_cached = true;
  return PS_OK;
}

int ps_weights(ps_game* G, int p, int normalized, float* out) {
  if (!G || !out) return fail(PS_ERR_INVALID, "null argument");
  const auto& v = normalized ? G->normalized[p & 1] : G->weights[p & 1];
  std::copy(v.begin(), v.end(), out);
  return PS_OK;
}

int ps_total_bet_amount(ps_game* G, int32_t out[2]) {
  if (!G) return fail(PS_ERR_INVALID, "null game");
  out[0] = G->total_bet[0];
  out[1] = G->total_bet[1];
  return PS_OK;
}

int ps_expected_values(ps_game* G, int player, int detail, float* out) {  // query.rs:639-760
  if (!G || !out || (player != 0 && player != 1)) return fail(PS_ERR_INVALID, "bad argument");
  if (G->state != GState::Solved) return fail(PS_ERR_STATE, "Game is not solved");
  if (!G->normalized_cached) return fail(PS_ERR_STATE, "Normalized weights are not cached");
  Game& g = *G->g;
  int rc = sync_host(G);
  if (rc) return rc;
  size_t idx = cur_index(G);
  const ArenaNode& n = g.arena[idx];
  const int H = g.H[player];
  int cf = 1;
  if (g.turn == NOT_DEALT && G->turn != NOT_DEALT) cf *= 45;
  if (g.river == NOT_DEALT && G->river != NOT_DEALT) cf *= 44;
  bool have_actions = false;
  float normalizer = (float)(g.num_combinations * (double)cf);
  std::vector<float> ret;
  if (n.terminal()) {
    normalizer = (float)g.num_combinations;
    Batch& B = *G->b;
    const int o = player ^ 1;
    std::vector<float> reach(g.hs[o], 0.f);
    std::copy(G->weights[o].begin(), G->weights[o].end(), reach.begin());
    CU(cudaMemcpyAsync(B.d_scratch, reach.data(), 4 * reach.size(), cudaMemcpyHostToDevice, B.stream));
    Op op{};
    op.type = OP_TERM;
    op.node = (uint32_t)idx;
    op.src = 0;
    op.dst = 1;
    op.board = (uint16_t)g.node_board[idx];
    op.term = n.boundary() ? TERM_BOUNDARY : n.fold() ? TERM_FOLD : TERM_SHOWDOWN;
    op.fold_pl = n.player & PL_MASK;
    if (n.boundary() && (rc = need_boundaries(G))) return rc;
    CU(cudaMemsetAsync(B.d_err, 0, sizeof(int), B.stream));
    CU(launch_eval_terminal(B.d_spots, op, player, B.d_scratch, B.scratch_floats, B.d_err, B.block, B.plan, B.stream));
    ret.resize(H);
    CU(cudaMemcpyAsync(ret.data(), B.d_scratch + g.vstride, 4 * (size_t)H, cudaMemcpyDeviceToHost, B.stream));
    CU(cudaStreamSynchronize(B.stream));
    if ((rc = B.check_err())) return rc;
  } else if (n.chance() && n.ch_off != 0xFFFFFFFFu && ((n.player & PL_MASK) ^ 1) == player) {
    ret.assign(G->hCH.begin() + n.ch_off, G->hCH.begin() + n.ch_off + H);
  } else if (!n.chance() && n.ip_off != 0xFFFFFFFFu && player == 1) {
    ret.assign(G->hIP.begin() + n.ip_off, G->hIP.begin() + n.ip_off + H);
  } else if (!n.chance() && player == n.player) {
    have_actions = true;
    ret.resize((size_t)n.nch * H);
    for (int a = 0; a < n.nch; ++a)
      for (int h = 0; h < H; ++h) ret[(size_t)a * H + h] = G->hR[n.rs_off + (size_t)a * g.hs[player] + h];
  } else {
    ret = G->cfv_cache[player];
  }
  int bias = std::max(G->total_bet[player] - G->total_bet[player ^ 1], 0);
  for (size_t a = 0; a * H < ret.size(); ++a) {
    bool is_fold = have_actions && g.arena[idx + n.child_off + a].prev.kind == ACT_FOLD;
    apply_swap(G, ret.data() + a * H, player, false);
    for (int h = 0; h < H; ++h) {
      float& v = ret[a * H + h];
      float wr = G->weights[player][h], wn = G->normalized[player][h];
      if (is_fold || wn == 0.0f) {
        v = 0.0f;
      } else {
        v *= normalizer * (wr / wn);
        v += (float)g.cfg.starting_pot * 0.5f + (float)(n.amount + bias);
      }
    }
  }
  if (!detail && !is_terminal(G) && !is_chance(G) && (int)n.player == player) {
    std::vector<float> st((size_t)n.nch * H);
    rc = ps_strategy(G, st.data());
    if (rc < 0) return rc;
    for (int h = 0; h < H; ++h) {
      float ev = 0.f;
      for (int a = 0; a < n.nch; ++a) ev += ret[h + (size_t)a * H] * st[h + (size_t)a * H];
      out[h] = ev;
    }
    return H;
  }
  std::copy(ret.begin(), ret.end(), out);
  return (int)ret.size();
}

// ---- checkpoint ----
int ps_state_export(ps_game* G, void* buf, uint64_t cap, uint64_t* needed) {
  if (!G || !needed) return fail(PS_ERR_INVALID, "null argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  Game& g = *G->g;
  uint64_t n = 16 + 8 * g.num_storage;
  *needed = n;
  if (!buf) return PS_OK;
  if (cap < n) return fail(PS_ERR_INVALID, "buffer too small");
  uint64_t hdr[2] = {0x3153505342303032ull, g.num_storage};
  std::memcpy(buf, hdr, 16);
  const SpotDev& s = G->b->h_spots[0];
  CU(cudaMemcpy((char*)buf + 16, s.S, 4 * g.num_storage, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy((char*)buf + 16 + 4 * g.num_storage, s.R, 4 * g.num_storage, cudaMemcpyDeviceToHost));
  return PS_OK;
}

int ps_state_import(ps_game* G, const void* buf, uint64_t size) {
  if (!G || !buf) return fail(PS_ERR_INVALID, "null argument");
  if (G->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  Game& g = *G->g;
  uint64_t hdr[2];
  if (size < 16) return fail(PS_ERR_INVALID, "storage size mismatch");
  std::memcpy(hdr, buf, 16);
  if (hdr[0] != 0x3153505342303032ull || hdr[1] != g.num_storage || size != 16 + 8 * g.num_storage)
    return fail(PS_ERR_INVALID, "storage size mismatch");
  const SpotDev& s = G->b->h_spots[0];
  CU(cudaMemcpy(s.S, (const char*)buf + 16, 4 * g.num_storage, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(s.R, (const char*)buf + 16 + 4 * g.num_storage, 4 * g.num_storage, cudaMemcpyHostToDevice));
  G->host_dirty = true;
  return PS_OK;
}

// ---- batch ----
struct ps_batch {
  std::unique_ptr<Batch> b;
};

int ps_batch_new(const ps_card_config* cards, const ps_tree_config* trees, int32_t n, const ps_batch_opts* opts,
                 ps_batch** out) {
  if (!cards || !trees || !out || n <= 0) return fail(PS_ERR_INVALID, "bad argument");
  *out = nullptr;
  auto B = std::make_unique<Batch>();
  B->games.resize(n);
  std::vector<std::string> errs(n);
  // tree construction is host work per spot: spread over the host cores
  int T = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  std::vector<int> ok(n, 0);
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t]() {
      for (int i = t; i < n; i += T) {
        TreeCfg tc;
        if (!parse_tree_config(&trees[i], tc, errs[i])) continue;
        auto g = std::make_unique<Game>();
        const ps_card_config& c = cards[i];
        uint8_t board[5] = {c.flop[0], c.flop[1], c.flop[2], c.turn, c.river};
        if (!c.range[0] || !c.range[1]) {
          errs[i] = "null range";
          continue;
        }
        if (!g->init(c.range[0], c.range[1], board, tc, errs[i])) continue;
        B->games[i] = std::move(g);
        ok[i] = 1;
      }
    });
  for (auto& x : th) x.join();
  for (int i = 0; i < n; ++i)
    if (!ok[i]) return fail(PS_ERR_INVALID, "spot " + std::to_string(i) + ": " + errs[i]);
  int rc = B->build(opts);
  if (rc) return rc;
  auto* pb = new ps_batch();
  pb->b = std::move(B);
  *out = pb;
  return PS_OK;
}

void ps_batch_free(ps_batch* b) { delete b; }

int ps_batch_solve(ps_batch* pb, uint32_t max_iter, const float* target) {
  if (!pb || !target) return fail(PS_ERR_INVALID, "bad argument");
  return pb->b->solve(max_iter, target, true);
}

int ps_batch_run_iterations(ps_batch* pb, uint32_t t0, uint32_t t1, int32_t epilogue) {
  if (!pb || t1 < t0 || t1 > (1u << 24) || (epilogue & ~(EPI_ROOT | EPI_EXPL)))
    return fail(PS_ERR_INVALID, "bad argument");
  return pb->b->run_iterations(t0, t1, epilogue);
}

int ps_batch_reset(ps_batch* pb) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  pb->b->ready = false;
  pb->b->h_expl.clear();
  return PS_OK;
}

int64_t ps_batch_num_boundary_items(ps_batch* pb) { return pb ? (int64_t)pb->b->items.size() : -1; }

int ps_batch_boundary_items(ps_batch* pb, int32_t* spot, int32_t* ordinal, uint8_t* boards, float* pots,
                            float* stacks) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  Batch& B = *pb->b;
  for (size_t i = 0; i < B.items.size(); ++i) {
    const Game& g = *B.games[B.items[i].x];
    if (spot) spot[i] = B.items[i].x;
    if (ordinal) ordinal[i] = B.items[i].y;
    if (boards) {
      const uint8_t bd[4] = {g.flop[0], g.flop[1], g.flop[2], g.turn};
      std::memcpy(boards + 4 * i, bd, 4);
    }
    // the boundary node's pot and the stack behind it (cfvnet neural_net_evaluator.rs:109-110)
    int64_t node = -1;
    for (size_t k = 0; k < g.bnd_ordinal.size(); ++k)
      if (g.bnd_ordinal[k] == B.items[i].y) node = (int64_t)k;
    const int amount = node >= 0 ? g.arena[node].amount : 0;
    if (pots) pots[i] = (float)(g.cfg.starting_pot + 2 * amount);
    if (stacks) stacks[i] = (float)(g.cfg.effective_stack - amount);
  }
  return PS_OK;
}

int ps_batch_set_boundary_cfvs(ps_batch* pb, const float* values, int32_t on_device) {
  if (!pb || !values) return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  const size_t ni = B.items.size();
  if (ni == 0) return PS_OK;
  const float* src = values;
  float* tmp = nullptr;
  if (!on_device) {
    CU(cudaMalloc(&tmp, 4 * ni * 2 * 1326));
    CU(cudaMemcpyAsync(tmp, values, 4 * ni * 2 * 1326, cudaMemcpyHostToDevice, B.stream));
    src = tmp;
  }
  std::unique_ptr<float, decltype(&cudaFree)> keep(tmp, &cudaFree);
  CU(launch_boundary_combo(B.d_spots, B.d_items, (int)ni, BC_SET_VALUES, src, nullptr, B.stream));
  CU(cudaStreamSynchronize(B.stream));
  return PS_OK;
}

int ps_batch_boundary_reach(ps_batch* pb, float* out, int32_t on_device) {
  if (!pb || !out) return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  const size_t ni = B.items.size();
  if (ni == 0) return PS_OK;
  float* dst = out;
  float* tmp = nullptr;
  if (!on_device) {
    CU(cudaMalloc(&tmp, 4 * ni * 2 * 1326));
    dst = tmp;
  }
  std::unique_ptr<float, decltype(&cudaFree)> keep(tmp, &cudaFree);
  CU(launch_boundary_combo(B.d_spots, B.d_items, (int)ni, BC_REACH, nullptr, dst, B.stream));
  if (!on_device) CU(cudaMemcpyAsync(out, tmp, 4 * ni * 2 * 1326, cudaMemcpyDeviceToHost, B.stream));
  CU(cudaStreamSynchronize(B.stream));
  return PS_OK;
}

int ps_batch_root_cfvalues_all(ps_batch* pb, float* out, int32_t on_device) {
  if (!pb || !out) return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  const size_t n = B.games.size(), bytes = 4 * n * 2 * 1326;
  float* dst = out;
  float* tmp = nullptr;
  if (!on_device) {
    CU(cudaMalloc(&tmp, bytes));
    dst = tmp;
  }
  std::unique_ptr<float, decltype(&cudaFree)> keep(tmp, &cudaFree);
  CU(launch_spot_combo(B.d_spots, (int)n, SC_ROOT, nullptr, dst, B.stream));
  if (!on_device) CU(cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, B.stream));
  CU(cudaStreamSynchronize(B.stream));
  return PS_OK;
}

int ps_batch_adjoint(ps_batch* pb, const float* cot, float* dw, float* dB, int32_t on_device) {
  if (!pb || !cot) return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  int rc = B.ensure_adjoint();
  if (rc) return rc;
  const size_t n = B.games.size(), ni = B.items.size();
  const size_t vb = 4 * n * 2 * 1326, ib = 4 * ni * 2 * 1326;
  const float* d_cot = cot;
  float* d_dw = dw;
  float* d_dB = dB;
  char* tmp = nullptr;
  if (!on_device) {
    CU(cudaMalloc(&tmp, 2 * vb + ib + 16));
    d_cot = (const float*)tmp;
    d_dw = dw ? (float*)(tmp + vb) : nullptr;
    d_dB = dB ? (float*)(tmp + 2 * vb) : nullptr;
    CU(cudaMemcpyAsync((void*)d_cot, cot, vb, cudaMemcpyHostToDevice, B.stream));
  }
  std::unique_ptr<char, decltype(&cudaFree)> keep(tmp, &cudaFree);
  CU(launch_spot_combo(B.d_spots, (int)n, SC_COT, d_cot, nullptr, B.stream));
  if ((rc = B.adjoint())) return rc;
  if (d_dw) CU(launch_spot_combo(B.d_spots, (int)n, SC_DW, nullptr, d_dw, B.stream));
  if (d_dB && ni) CU(launch_boundary_combo(B.d_spots, B.d_items, (int)ni, BC_GRAD, nullptr, d_dB, B.stream));
  if (!on_device) {
    if (dw) CU(cudaMemcpyAsync(dw, d_dw, vb, cudaMemcpyDeviceToHost, B.stream));
    if (dB && ni) CU(cudaMemcpyAsync(dB, d_dB, ib, cudaMemcpyDeviceToHost, B.stream));
  }
  CU(cudaStreamSynchronize(B.stream));
  return PS_OK;
}

int64_t ps_batch_record_bytes(ps_batch* pb) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  if (pb->b->board_size() < 0) return fail(PS_ERR_INVALID, "records of one batch need one board size");
  return (int64_t)pb->b->record_bytes();
}

int ps_batch_records(ps_batch* pb, uint8_t* out, int32_t on_device) {
  if (!pb || !out) return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  const size_t bytes = B.record_bytes();
  if (bytes == 0) return fail(PS_ERR_INVALID, "records of one batch need one board size");
  uint8_t* dst = out;
  uint8_t* tmp = nullptr;
  if (!on_device) {
    CU(cudaMalloc(&tmp, bytes));
    dst = tmp;
  }
  std::unique_ptr<uint8_t, decltype(&cudaFree)> keep(tmp, &cudaFree);
  int rc = B.records(dst);
  if (rc) return rc;
  if (!on_device) CU(cudaMemcpy(out, tmp, bytes, cudaMemcpyDeviceToHost));
  return PS_OK;
}

int ps_sample_situations(const ps_sampler_config* cfg, int64_t first, int32_t n, uint8_t* boards, int32_t* pots,
                         int32_t* stacks, float* ranges, void* stream) {
  if (!cfg || n < 0 || first < 0 || (n > 0 && (!boards || !pots || !stacks || !ranges)))
    return fail(PS_ERR_INVALID, "bad argument");
  if (cfg->board_size != 4 && cfg->board_size != 5) return fail(PS_ERR_INVALID, "board_size must be 4 or 5");
  if (cfg->num_pot_intervals < 1 || cfg->num_pot_intervals > kMaxSamplerIntervals || !cfg->pot_intervals ||
      cfg->num_spr_intervals < 0 || cfg->num_spr_intervals > kMaxSamplerIntervals ||
      (cfg->num_spr_intervals > 0 && !cfg->spr_intervals))
    return fail(PS_ERR_INVALID, "1 to 16 pot intervals and 0 to 16 SPR intervals");
  if (cfg->initial_stack <= 0) return fail(PS_ERR_INVALID, "initial_stack must be > 0");
  SamplerParams P{};
  P.board_size = cfg->board_size;
  P.initial_stack = cfg->initial_stack;
  P.npot = cfg->num_pot_intervals;
  P.nspr = cfg->num_spr_intervals;
  for (int k = 0; k < P.npot; ++k) {
    P.pot[k][0] = cfg->pot_intervals[2 * k];
    P.pot[k][1] = cfg->pot_intervals[2 * k + 1];
    if (P.pot[k][0] < 1 || P.pot[k][1] <= P.pot[k][0]) return fail(PS_ERR_INVALID, "pot intervals need 1 <= lo < hi");
  }
  for (int k = 0; k < P.nspr; ++k) {
    P.spr[k][0] = cfg->spr_intervals[2 * k];
    P.spr[k][1] = cfg->spr_intervals[2 * k + 1];
    if (!(P.spr[k][0] >= 0.0) || !(P.spr[k][1] > P.spr[k][0]) || P.spr[k][1] > 1e6)
      return fail(PS_ERR_INVALID, "SPR intervals need 0 <= lo < hi");
  }
  P.seed = cfg->seed;
  P.first = first;
  if (n == 0) return PS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  StagingLease lease;
  CU(lease.acquire(sizeof(int)));
  lease.using_stream(s);
  int* d_err = (int*)lease.ptr;
  CU(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  CU(launch_sample_situations(P, n, boards, pots, stacks, ranges, d_err, s));
  int e = 0;
  CU(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  lease.done();
  if (e)
    return fail(PS_ERR_INVALID, "a situation could not be drawn: pot and SPR intervals infeasible for the initial "
                                "stack (10000 attempts, as the reference)");
  return PS_OK;
}

int ps_boundary_encode(int32_t n, const uint8_t* boards, const float* pots, const float* stacks, const float* reach,
                       void* out, int32_t out_bf16, void* stream) {
  if (n < 0 || (n > 0 && (!boards || !pots || !stacks || !reach || !out)))
    return fail(PS_ERR_INVALID, "bad argument");
  if (n == 0) return PS_OK;
  std::vector<uint8_t> hb((size_t)n * 4);
  for (int i = 0; i < n; ++i) {
    uint64_t seen = 0;
    for (int k = 0; k < 4; ++k) {
      const uint8_t c = boards[4 * i + k];
      if (c >= 52 || (seen >> c & 1)) return fail(PS_ERR_INVALID, "boards must hold 4 distinct cards below 52");
      seen |= 1ull << c;
      hb[4 * i + k] = c;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  const size_t ob = ((hb.size() + 15) & ~(size_t)15);
  StagingLease lease;
  CU(lease.acquire(ob + 8 * (size_t)n + 16));
  lease.using_stream(s);
  char* d = lease.ptr;
  float* d_pot = (float*)(d + ob);
  float* d_stack = d_pot + n;
  CU(cudaMemcpyAsync(d, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d_pot, pots, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d_stack, stacks, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
  CU(launch_boundary_encode(n, (const uint8_t*)d, d_pot, d_stack, reach, out, out_bf16 ? 1 : 0, s));
  CU(cudaStreamSynchronize(s));
  lease.done();
  return PS_OK;
}

int ps_batch_results(ps_batch* pb, float* expl, int32_t* iters) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  Batch& B = *pb->b;
  if (B.h_expl.empty()) return fail(PS_ERR_STATE, "batch not solved");
  if (expl) std::copy(B.h_expl.begin(), B.h_expl.end(), expl);
  if (iters) std::copy(B.h_iters.begin(), B.h_iters.end(), iters);
  return PS_OK;
}

int ps_batch_root_strategy(ps_batch* pb, int32_t spot, float* out) {
  if (!pb || spot < 0 || spot >= (int)pb->b->games.size()) return fail(PS_ERR_INVALID, "bad spot");
  Batch& B = *pb->b;
  Game& g = *B.games[spot];
  size_t root = 0;
  while (!g.arena[root].terminal() && !g.arena[root].chance() && g.arena[root].nch == 1) root += g.arena[root].child_off;
  const ArenaNode& n = g.arena[root];
  int p = n.player, H = g.H[p], hs = g.hs[p], na = n.nch;
  std::vector<float> S((size_t)na * hs);
  CU(cudaMemcpy(S.data(), B.h_spots[spot].S + n.rs_off, 4 * S.size(), cudaMemcpyDeviceToHost));
  float def = 1.0f / (float)na;
  for (int h = 0; h < H; ++h) {
    float d = S[h];
    for (int a = 1; a < na; ++a) d += S[(size_t)a * hs + h];
    for (int a = 0; a < na; ++a) out[(size_t)a * H + h] = d == 0.0f ? def : S[(size_t)a * hs + h] / d;
  }
  return na * H;
}

int64_t ps_batch_num_nodes(ps_batch* pb, int32_t spot) {
  if (!pb || spot < 0 || spot >= (int)pb->b->games.size()) return fail(PS_ERR_INVALID, "bad spot");
  return (int64_t)pb->b->games[spot]->arena.size();
}

int64_t ps_batch_node_storage(ps_batch* pb, int32_t spot, int64_t node, int which, float* out) {
  if (!pb || !out || spot < 0 || spot >= (int)pb->b->games.size() || (which != 1 && which != 2))
    return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  const Game& g = *B.games[spot];
  if (node < 0 || node >= (int64_t)g.arena.size()) return fail(PS_ERR_INVALID, "bad node index");
  const ArenaNode& n = g.arena[node];
  if (n.terminal() || n.chance()) return 0;
  const int p = n.player, H = g.H[p], hs = g.hs[p];
  const float* src = (which == 1 ? B.h_spots[spot].S : B.h_spots[spot].R) + n.rs_off;
  std::vector<float> rows((size_t)n.nch * hs);
  CU(cudaMemcpy(rows.data(), src, 4 * rows.size(), cudaMemcpyDeviceToHost));
  for (int a = 0; a < n.nch; ++a)
    std::copy(rows.begin() + (size_t)a * hs, rows.begin() + (size_t)a * hs + H, out + (size_t)a * H);
  return (int64_t)n.nch * H;
}

int ps_batch_root_cfvalues(ps_batch* pb, int32_t spot, int player, float* out) {
  if (!pb || !out || spot < 0 || spot >= (int)pb->b->games.size() || (player != 0 && player != 1))
    return fail(PS_ERR_INVALID, "bad argument");
  Batch& B = *pb->b;
  const int H = B.games[spot]->H[player];
  CU(cudaMemcpy(out, B.h_spots[spot].root_out[player], 4 * (size_t)H, cudaMemcpyDeviceToHost));
  return H;
}

int ps_batch_last_timing(ps_batch* pb, float* solve_ms, float* setup_ms) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  if (solve_ms) *solve_ms = pb->b->last_solve_ms;
  if (setup_ms) *setup_ms = pb->b->last_setup_ms;
  return PS_OK;
}

double ps_batch_iteration_bytes(ps_batch* pb, int32_t spot) {
  if (!pb || spot < 0 || spot >= (int)pb->b->games.size()) return -1.0;
  Game& g = *pb->b->games[spot];
  double s = 0;
  for (const auto& n : g.arena)
    if (!n.terminal() && !n.chance() && n.nch > 1) s += (double)n.nch * g.H[n.player];
  return 20.0 * s;
}

int ps_batch_io_bytes(ps_batch* pb, uint64_t* h2d, uint64_t* d2h) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  Batch& B = *pb->b;
  const size_t n = B.games.size();
  if (h2d) *h2d = B.static_bytes + n * (sizeof(SpotDev) + sizeof(int) + sizeof(float)) + (size_t)B.nwork * sizeof(int2);
  if (d2h) *d2h = n * (sizeof(float) + sizeof(int));
  return PS_OK;
}

int ps_batch_scan_buffers(ps_batch* pb) { return pb ? pb->b->plan.bufs : fail(PS_ERR_INVALID, "null batch"); }

int ps_batch_config(ps_batch* pb, int32_t* block, int32_t* grid, int32_t* cps) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  const Batch& B = *pb->b;
  if (block) *block = B.flow ? B.flow_block : B.block;
  if (grid) *grid = B.flow ? B.flow_grid : B.grid;
  if (cps) *cps = B.flow ? B.flow_cps : B.ctas_per_sm;
  return PS_OK;
}

static void schedule_of(const Batch& B, int32_t out[8]) {
  out[0] = B.flow ? PS_SCHED_FLOW : PS_SCHED_STEP;
  out[1] = B.flow ? B.flow_block : B.block;
  out[2] = B.flow ? B.flow_grid : B.grid;
  out[3] = B.flow ? B.flow_cps : B.ctas_per_sm;
  out[4] = B.flow ? B.flow_plan.bufs : B.plan.bufs;
  out[5] = B.flow ? B.flow_lanes : B.inst_k;
  out[6] = B.flow ? B.flow_parts : 1;
  out[7] = B.grid_mode ? (B.grid_cluster ? 2 : 1) : 0;
}

int ps_batch_schedule(ps_batch* pb, int32_t out[8]) {
  if (!pb || !out) return fail(PS_ERR_INVALID, "null argument");
  schedule_of(*pb->b, out);
  return PS_OK;
}

int ps_game_schedule(ps_game* g, int32_t out[8]) {
  if (!g || !out) return fail(PS_ERR_INVALID, "null argument");
  if (g->state == GState::TreeBuilt) return fail(PS_ERR_STATE, "Memory is not allocated");
  schedule_of(*g->b, out);
  if (g->b->grid_mode) out[2] = g->b->grid_blocks;
  return PS_OK;
}

int ps_batch_autotune_trials(ps_batch* pb, int32_t* shape, float* trial_ms, int cap) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  const auto& L = pb->b->tune_log;
  for (int i = 0; i < (int)L.size() && i < cap; ++i) {
    if (shape) {
      shape[4 * i] = L[i].block;
      shape[4 * i + 1] = L[i].bufs;
      shape[4 * i + 2] = L[i].lanes;
      shape[4 * i + 3] = L[i].parts;
    }
    if (trial_ms) trial_ms[i] = L[i].ms;
  }
  return (int)L.size();
}

int ps_batch_autotune_log(ps_batch* pb, int32_t* block_threads, int32_t* scan_buffers, float* trial_ms, int cap) {
  if (!pb) return fail(PS_ERR_INVALID, "null batch");
  const auto& L = pb->b->tune_log;
  for (int i = 0; i < (int)L.size() && i < cap; ++i) {
    if (block_threads) block_threads[i] = L[i].block;
    if (scan_buffers) scan_buffers[i] = L[i].bufs;
    if (trial_ms) trial_ms[i] = L[i].ms;
  }
  return (int)L.size();
}

}  // extern "C"

// ---- test hooks ----
int ps_debug_grid_barrier_timeout(int32_t ctas, int32_t rounds, int64_t wait_ns, int32_t all_join, int32_t* err,
                                  int32_t* passed, float* ms) {
  if (!err || !passed || !ms || ctas < 2 || rounds < 1 || wait_ns < 0 || wait_ns > 1000000000LL)
    return fail(PS_ERR_INVALID, "bad argument");
  DeviceConsts* dc = nullptr;
  int rc = device_consts(&dc);
  if (rc) return rc;
  char* d = nullptr;
  CU(cudaMalloc(&d, 64));
  std::unique_ptr<char, decltype(&cudaFree)> keep(d, &cudaFree);
  unsigned* bar = (unsigned*)d;
  int* d_err = (int*)(d + 16);
  int* d_passed = (int*)(d + 20);
  cudaStream_t s = nullptr;
  CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  std::unique_ptr<CUstream_st, decltype(&cudaStreamDestroy)> ks(s, &cudaStreamDestroy);
  cudaEvent_t ev[2];
  CU(cudaEventCreate(&ev[0]));
  CU(cudaEventCreate(&ev[1]));
  CU(cudaMemsetAsync(d + 16, 0, 8, s));
  CU(cudaEventRecord(ev[0], s));
  CU(launch_debug_barrier_timeout(ctas, rounds, wait_ns, all_join, bar, d_err, d_passed, s));
  CU(cudaEventRecord(ev[1], s));
  int h[2] = {0, 0};
  CU(cudaMemcpyAsync(h, d + 16, 8, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  CU(cudaEventElapsedTime(ms, ev[0], ev[1]));
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  *err = h[0];
  *passed = h[1];
  return PS_OK;
}
