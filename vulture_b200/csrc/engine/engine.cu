// engine.cu -- the vgpu C ABI (include/vgpu.h) on one B200.
//
// vgpu_create uploads a vgpu_problem into device memory (fields and
// coefficients as padded [n0][n1][n2p] volumes, k rows aligned to 32
// elements), builds the launch plan of one time step in the reference's order
// (src/simulation.c:156-222), and captures runs of steps in CUDA graphs.
// vgpu_run replays the graphs; the running DFT of the frequency-domain
// observers is accumulated every chunk from a buffer of field samples.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>

#include "kernels.cuh"
#include "sweep_tma.cuh"

#include <cudaTypedefs.h>

using namespace vgpu_dev;

static thread_local char g_err[1024];

static int set_err(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

extern "C" const char *vgpu_last_error(void) { return g_err; }

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return set_err(VGPU_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

static const int kChunk = 64;      // steps per block and per DFT block
static const int kTwRows = kChunk; // twiddle rows of one DFT fold (one block)
// DFT staging rows: two blocks' worth, so that the sample of a block's first
// step, taken at the end of the previous block (merged side launch), never
// lands on a row that block's fold has yet to read.
static const int kStageRows = 2 * kChunk;
static const int kGraphSteps = 16; // steps of the longest step graph; a full block replays it kChunk / kGraphSteps times

// The device step counter moves once per block of steps; kernels inside
// the block add their step's offset (step_rel).
__global__ void k_advance(uint64_t *step, int nsteps) { *step += nsteps; }

// Device memory of destroyed engines is kept in a per-device cache and
// handed to later engines that ask for a block of about the same size, so
// that creating a problem again (tests, batches, a service) does not map new
// pages.  The cache gives its memory back to the driver when it holds more
// than a quarter of the device, and when an allocation would not fit.
struct BlockCache {
  std::mutex mu;
  std::map<int, std::multimap<size_t, void *>> free_blocks;   // device -> size -> block
  std::map<int, size_t> held;

  // A cached block of at least b bytes (and not much more), or null; its
  // size goes to *got.
  void *take(int dev, size_t b, size_t *got)
  {
    std::lock_guard<std::mutex> lk(mu);
    auto &fb = free_blocks[dev];
    auto it = fb.lower_bound(b);
    if (it == fb.end() || it->first > 2 * b + (1u << 20)) return nullptr;
    void *p = it->second;
    *got = it->first;
    held[dev] -= it->first;
    fb.erase(it);
    return p;
  }
  // Takes back n blocks; past a quarter of the device's memory the cache
  // is released.
  void give(int dev, size_t n, const size_t *b, void *const *p)
  {
    std::lock_guard<std::mutex> lk(mu);
    size_t total = 0, fr = 0;
    cudaMemGetInfo(&fr, &total);
    for (size_t q = 0; q < n; q++) {
      free_blocks[dev].emplace(b[q], p[q]);
      held[dev] += b[q];
    }
    if (held[dev] > total / 4) release_locked(dev);
  }
  void release(int dev)
  {
    std::lock_guard<std::mutex> lk(mu);
    release_locked(dev);
  }
  void release_locked(int dev)
  {
    for (auto &kv : free_blocks[dev]) cudaFree(kv.second);
    free_blocks[dev].clear();
    held[dev] = 0;
  }
};

// Engines being created at this moment, process-wide: a creation's host
// threads share the cores with the others'.
static std::atomic<int> g_creating{ 0 };

static int host_threads()
{
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int busy = std::max(1, g_creating.load());
  return std::max(1, std::min(32, hw / busy));
}

// Host threads for set-up and read-back work, started once and kept: a
// thread started per parallel section costs tens of microseconds, more than
// the section's work on a small mesh, and a creation or read-back has tens
// of sections.  run(n, fn) calls fn(0 .. n-1) on the pool and the calling
// thread and returns when all have returned.  One section runs at a time
// (creations on several threads take turns with their sections); a section
// started from inside a section runs on the calling thread alone.
class HostPool {
 public:
  static HostPool &get()
  {
    static HostPool *p = new HostPool();   // never destroyed: its threads live until exit
    return *p;
  }
  int size() const { return (int)threads_.size() + 1; }
  template <typename F>
  void run(int n, F &&fn)
  {
    if (n <= 0) return;
    if (n == 1 || in_section()) {
      for (int w = 0; w < n; w++) fn(w);
      return;
    }
    std::lock_guard<std::mutex> section(run_mu_);
    std::function<void(int)> job = fn;
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &job;
      n_ = n;
      next_ = 0;
      left_ = n;
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return left_ == 0; });
    job_ = nullptr;
  }

 private:
  HostPool()
  {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    for (int q = 1; q < std::min(hw, 32); q++) threads_.emplace_back([this] { loop(); });
    for (auto &t : threads_) t.detach();
  }
  static bool &in_section()
  {
    static thread_local bool f = false;
    return f;
  }
  // Take items of the current section until none is left.
  void work()
  {
    in_section() = true;
    for (;;) {
      int w;
      const std::function<void(int)> *job;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!job_ || next_ >= n_) break;
        w = next_++;
        job = job_;
      }
      (*job)(w);
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_cv_.notify_all();
    }
    in_section() = false;
  }
  void loop()
  {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      work();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)> *job_ = nullptr;
  int n_ = 0, next_ = 0, left_ = 0;
  uint64_t gen_ = 0;
};

// Run fn(lo, hi) over [0, n) split into contiguous ranges on up to
// host_threads() pool threads (the calling thread takes part).
template <typename F>
static void parallel_ranges(size_t n, F fn, size_t min_per_thread = 256)
{
  const size_t nthr = std::max<size_t>(
      1, std::min<size_t>(std::min<size_t>((size_t)host_threads(), (size_t)HostPool::get().size()), n / min_per_thread));
  if (nthr <= 1) {
    fn((size_t)0, n);
    return;
  }
  HostPool::get().run((int)nthr, [&](int w) { fn(n * w / nthr, n * (w + 1) / nthr); });
}

static BlockCache &block_cache()
{
  static BlockCache *c = new BlockCache();   // never destroyed: it may outlive the CUDA runtime at exit
  return *c;
}

// Pinned host staging for large device-to-host reads.  A read into pageable
// memory runs at a fraction of the link's speed (the driver stages it
// itself, one core copying into freshly faulted pages); here it goes
// through two pinned chunks, the DMA of one overlapping the host copy of the
// other, which runs on several threads.  The first engine created pins the
// chunks, once per process.  (Uploads at creation stay plain
// asynchronous copies: staging them needs a stream synchronisation per copy,
// which made creating 256 batch engines 3.4x slower.)  One pair serves the process
// (portable across devices), under a lock; it is allocated by the first
// engine that needs it and kept until exit.
// Host copy of n bytes on up to 8 threads (large copies into fresh pages
// are bound by page faults and one core's copy rate).
static void host_copy(void *dst, const void *src, size_t n)
{
  const size_t parts = std::min<size_t>((size_t)HostPool::get().size(), std::max<size_t>(1, n >> 20));   // 1 MB or more each
  if (parts <= 1) {
    memcpy(dst, src, n);
    return;
  }
  HostPool::get().run((int)parts, [=](int w) {
    const size_t a = n * w / parts, b = n * (w + 1) / parts;
    memcpy((char *)dst + a, (const char *)src + a, b - a);
  });
}

struct PinnedStage {
  static constexpr size_t kChunkBytes = 16u << 20;
  std::mutex mu;
  char *buf = nullptr;

  int ensure_locked()
  {
    std::lock_guard<std::mutex> lock(mu);
    return ensure();
  }

  int ensure()
  {
    if (buf) return 0;
    CK(cudaHostAlloc((void **)&buf, 2 * kChunkBytes, cudaHostAllocPortable));
    return 0;
  }

  // Device -> host: chunk q lands in half q % 2; while it is copied out on
  // the host, chunk q + 1 is in flight.
  int d2h(void *dst, const void *src, size_t bytes, cudaStream_t st)
  {
    std::lock_guard<std::mutex> lock(mu);
    if (int rc = ensure()) return rc;
    cudaEvent_t ev[2];
    CK(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    const size_t nchunks = (bytes + kChunkBytes - 1) / kChunkBytes;
    cudaError_t e = cudaSuccess;
    auto issue = [&](size_t q) {
      const size_t off = q * kChunkBytes, n = std::min(kChunkBytes, bytes - off);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + (q % 2) * kChunkBytes, (const char *)src + off, n, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaEventRecord(ev[q % 2], st);
    };
    if (nchunks) issue(0);
    for (size_t q = 0; q < nchunks && e == cudaSuccess; q++) {
      if (q + 1 < nchunks) issue(q + 1);
      if (e == cudaSuccess) e = cudaEventSynchronize(ev[q % 2]);
      if (e != cudaSuccess) break;
      const size_t off = q * kChunkBytes, n = std::min(kChunkBytes, bytes - off);
      host_copy((char *)dst + off, buf + (q % 2) * kChunkBytes, n);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // nothing of ours left in flight
    else cudaStreamSynchronize(st);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (e != cudaSuccess) return set_err(VGPU_ECUDA, "staged device-to-host copy: %s", cudaGetErrorString(e));
    return 0;
  }

};

// Pinned host arenas for the uploads of an engine's creation, kept for the
// process and shared by creations one at a time each: a large upload is
// copied into the creation's arena (on the host pool) and sent from there at
// the link's speed, and the arena is handed back once the creation's set-up
// stream has drained.  A pageable upload goes through the driver's own
// staging, one core at a time (about 7 GB/s here).
struct PinnedArenas {
  static constexpr size_t kArena = 128u << 20;
  std::mutex mu;
  std::vector<char *> free_list;
  char *take()
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!free_list.empty()) {
      char *a = free_list.back();
      free_list.pop_back();
      return a;
    }
    char *a = nullptr;
    if (cudaHostAlloc((void **)&a, kArena, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return a;
  }
  void give(char *a)
  {
    if (!a) return;
    std::lock_guard<std::mutex> lk(mu);
    free_list.push_back(a);
  }
};

static PinnedArenas &pinned_arenas()
{
  static PinnedArenas *a = new PinnedArenas;   // never destroyed: outlives every engine
  return *a;
}

// Page-locked host blocks for read-backs (vgpu_host_alloc), cached for the
// process: pinning costs milliseconds per megabyte, so a freed block is kept
// for the next request of about its size, up to 2 GB in all.
struct HostBlocks {
  static constexpr size_t kCacheMax = (size_t)2 << 30;
  std::mutex mu;
  std::multimap<size_t, void *> free_blocks;
  std::map<void *, size_t> sizes;   // every block handed out or cached
  size_t cached = 0;
  void *alloc(size_t b)
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = free_blocks.lower_bound(b);
    if (it != free_blocks.end() && it->first <= 2 * b + ((size_t)1 << 20)) {
      void *q = it->second;
      cached -= it->first;
      free_blocks.erase(it);
      return q;
    }
    void *q = nullptr;
    if (cudaHostAlloc(&q, b ? b : 1, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    sizes[q] = b;
    return q;
  }
  void release(void *q)
  {
    std::lock_guard<std::mutex> lk(mu);
    auto s = sizes.find(q);
    if (s == sizes.end()) return;
    free_blocks.emplace(s->second, q);
    cached += s->second;
    while (cached > kCacheMax && !free_blocks.empty()) {
      auto big = std::prev(free_blocks.end());
      cudaFreeHost(big->second);
      cached -= big->first;
      sizes.erase(big->second);
      free_blocks.erase(big);
    }
  }
};

static HostBlocks &host_blocks()
{
  static HostBlocks *h = new HostBlocks;   // never destroyed: outlives every engine
  return *h;
}

// Whether host memory is page-locked (a read into it needs no staging).
static bool is_pinned(const void *ptr)
{
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

static PinnedStage &pinned_stage()
{
  static PinnedStage *st = new PinnedStage;   // never destroyed: outlives every engine
  return *st;
}

struct DevAlloc {
  struct Block {
    void *p;
    size_t b;
  };
  std::vector<Block> blocks;
  uint64_t bytes = 0;
  int dev = -1;
  template <typename U>
  int alloc(U **p, size_t count)
  {
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return set_err(VGPU_ENODEV, "no CUDA device");
    const size_t b = (sizeof(U) * (count ? count : 1) + 255) / 256 * 256;
    size_t got = b;
    void *q = block_cache().take(dev, b, &got);
    if (!q) {
      cudaError_t e = cudaMalloc(&q, b);
      if (e != cudaSuccess) {
        cudaGetLastError();
        block_cache().release(dev);
        e = cudaMalloc(&q, b);
      }
      if (e != cudaSuccess) return set_err(VGPU_ENOMEM, "cudaMalloc of %zu bytes failed: %s", b, cudaGetErrorString(e));
    }
    *p = (U *)q;
    blocks.push_back(Block{ q, got });
    bytes += got;
    return 0;
  }
  void free_all()
  {
    std::vector<size_t> b;
    std::vector<void *> q;
    for (const Block &bl : blocks) {
      b.push_back(bl.b);
      q.push_back(bl.p);
    }
    if (!blocks.empty()) block_cache().give(dev, b.size(), b.data(), q.data());
    blocks.clear();
  }
};

struct EngineBase {
  virtual ~EngineBase() {}
  virtual int run(uint64_t n) = 0;
  virtual int read_td(double *out, uint64_t steps) = 0;
  virtual int read_dft(double *re, double *im) = 0;
  virtual int read_field(int c, double *out) = 0;
  virtual int write_field(int c, const double *in) = 0;
  virtual int check_finite() = 0;
  virtual int time_kernel(int kernel, int warmup, int iters, double *ms, uint64_t *points) = 0;
  virtual int sweep_points(int kernel, uint64_t *bulk_pts, uint64_t *pml_pts) = 0;
  virtual int check_steps(uint64_t nsteps) = 0;
  virtual int enqueue(uint64_t max_steps, uint64_t *queued) = 0;
  virtual int query() = 0;
  virtual int synchronize() = 0;
  vgpu_bin_sink bin_sink = nullptr;
  void *bin_user = nullptr;
  uint64_t step = 0;
  vgpu_stats stats{};
};

struct SrcLaunch {
  Box b;
  int c, kind;
  double soft;
  void *values;
};

template <typename T>
struct PwLaunch {
  PwView<T> pv;
  TfsfView te, th;
  int64_t total_e = 0, total_h = 0;
  TfsfList<T> le{}, lh{};   // point lists of the E and H corrections
};

// ---- host-side box helpers and the sweep plan --------------------------

static Box unite(const Box b[3])
{
  Box u{ 1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30) };
  for (int c = 0; c < 3; c++) {
    if (b[c].empty()) continue;
    u.i0 = std::min(u.i0, b[c].i0); u.i1 = std::max(u.i1, b[c].i1);
    u.j0 = std::min(u.j0, b[c].j0); u.j1 = std::max(u.j1, b[c].j1);
    u.k0 = std::min(u.k0, b[c].k0); u.k1 = std::max(u.k1, b[c].k1);
  }
  return u;
}

static bool boxes_meet(const Box &u, const Box &v)
{
  return !u.empty() && !v.empty() && u.i0 <= v.i1 && v.i0 <= u.i1 && u.j0 <= v.j1 && v.j0 <= u.j1 && u.k0 <= v.k1 &&
         v.k0 <= u.k1;
}

static int64_t box_overlap(const Box &u, const Box &v)
{
  if (!boxes_meet(u, v)) return 0;
  Box x{ std::max(u.i0, v.i0), std::min(u.i1, v.i1), std::max(u.j0, v.j0),
         std::min(u.j1, v.j1), std::max(u.k0, v.k0), std::min(u.k1, v.k1) };
  return x.count();
}

static Box tile_box(const SweepTile &t)
{
  return Box{ t.i0, t.i1, t.j0, t.j0 + kSweepJH - 1, t.k0, t.k0 + kSweepKW - 1 };
}

// The UPML regions of a problem: region q is outer face face[q], with the
// update limits lim[q][field] (src/pml.c:44-84).
struct RegionSet {
  int nreg = 0;
  int face[6] = {};
  Box lim[6][6];
};

static RegionSet regions_of(const vgpu_problem &p)
{
  RegionSet rs;
  for (int r = 0; r < 6; r++) {
    if (!p.pml_present[r]) continue;
    const int q = rs.nreg++;
    rs.face[q] = r;
    for (int f = 0; f < 6; f++) rs.lim[q][f] = box_from(p.pml_flim[r][f]);
  }
  return rs;
}

// The normal H of a Mur face (src/mur.c:401-555) takes the bulk H update
// (src/grid.c:800-888): the same expression, reading only E, at points the
// bulk limits leave out.  Where a face's box and its component's bulk box
// are disjoint and their union is itself a box (the face box extends the
// bulk box by a plane, as on every outer Mur face), the bulk box grows by
// it and the face needs no update of its own.  The reference updates Mur H
// before the bulk H; both read E only and write disjoint points, so the
// order does not matter.  Returns the bits of the faces absorbed.
static unsigned fold_mur_h(const vgpu_problem &p, Box bh[3])
{
  unsigned folded = 0;
  for (int pass = 0; pass < 2; pass++)   // a face may extend a box another face already grew
    for (int f = 0; f < 6; f++) {
      if (!p.mur_present[f] || (folded >> f & 1u)) continue;
      const int c = f / 2;                      // the face's normal H component
      const Box m = box_from(p.mur_flim[f][HX + c]);
      if (m.empty()) { folded |= 1u << f; continue; }
      Box &b = bh[c];
      if (b.empty() || boxes_meet(b, m)) continue;
      const Box u{ std::min(b.i0, m.i0), std::max(b.i1, m.i1), std::min(b.j0, m.j0), std::max(b.j1, m.j1),
                   std::min(b.k0, m.k0), std::max(b.k1, m.k1) };
      if (u.count() != b.count() + m.count()) continue;
      b = u;
      folded |= 1u << f;
    }
  return folded;
}

// The tiles of one half step (host only).  Columns of 32 x 8 points, cut
// into runs of i planes sized so a launch has several tiles per resident
// block (the pipeline runs across tile boundaries).  Bulk-footprint tiles
// whose rows reach into a Z region (the thin UPML slabs at the k ends) carry
// both the bulk box and the Z region; the X and Y regions get their own
// tiles.  With UPML regions, one launch of the UPML kernel takes every tile,
// bulk tiles interleaved evenly with the UPML and mixed ones: a block's
// memory-bound bulk tiles and issue-bound UPML tiles overlap on the SM,
// where two launches ran one after the other (graded 200x160x120 UPML mesh,
// FP32: step 153 -> 148 us).  halo: elements per 16 bytes of the storage
// type; nsm: SMs.
struct SweepPlan {
  std::vector<SweepTile> bulk, pml;   // the bulk kernel's and the UPML kernel's tiles
  int wn = 0;                         // width of the narrow auxiliary boxes (0: unused)
};

// Sweep tuning for the engines a thread creates and the groups it runs
// (vgpu_set_sweep_tuning): planes per tile (0: the size rule below), a cap
// on resident blocks per SM (0: as many as fit) and the tiles a grouped
// sweep block takes at a time (0: 4).
static thread_local int g_tune_depth = 0, g_tune_blocks = 0, g_tune_chunk = 0;

static SweepPlan plan_sweep(const Box &ub, const RegionSet &rs, bool es, int halo, int nsm, int depth = 0)
{
  SweepPlan pl;
  // Planes per tile: about 16 tiles per SM over the update box, 4 to 32.
  auto run_len = [&](int64_t cells) {
    if (depth > 0) return std::min(depth, kSweepMaxPlanes);
    int64_t t = cells / (256LL * nsm * 16);
    return (int)std::max<int64_t>(4, std::min<int64_t>(kSweepMaxPlanes, t));
  };
  std::vector<SweepTile> &bulk = pl.bulk, &pml = pl.pml;
  int wn = 0;
  Box zun[2];
  int zreg[2] = { -1, -1 }, nz = 0;
  Box core = ub;
  for (int q = 0; q < rs.nreg; q++) {
    Box c3[3] = { rs.lim[q][es ? EX : HX], rs.lim[q][es ? EY : HY], rs.lim[q][es ? EZ : HZ] };
    Box u = unite(c3);
    if (u.i1 < u.i0) continue;
    if (rs.face[q] / 2 == 2) {
      zun[nz] = u;
      zreg[nz++] = q;
      if (core.empty()) core = u;
      core = Box{ std::min(core.i0, u.i0), std::max(core.i1, u.i1), std::min(core.j0, u.j0),
                  std::max(core.j1, u.j1), std::min(core.k0, u.k0), std::max(core.k1, u.k1) };
    } else {
      const int ti = run_len(u.count());
      for (int i = u.i0; i <= u.i1; i += ti)
        for (int j = u.j0; j <= u.j1; j += kSweepJH)
          for (int k = (u.k0 / kSweepKW) * kSweepKW; k <= u.k1; k += kSweepKW)
            pml.push_back(SweepTile{ { q, -1 }, 0, i, std::min(i + ti - 1, u.i1), j, k, -1 });
    }
  }
  if (!core.empty()) {
    const int ti = run_len(core.count());
    for (int i = core.i0; i <= core.i1; i += ti)
      for (int j = core.j0; j <= core.j1; j += kSweepJH)
        for (int k = (core.k0 / kSweepKW) * kSweepKW; k <= core.k1; k += kSweepKW) {
          SweepTile t{ { -1, -1 }, 1, i, std::min(i + ti - 1, core.i1), j, k, -1 };
          const Box tb = tile_box(t);
          int r = 0, zi = -1;
          for (int z = 0; z < nz; z++)
            if (boxes_meet(tb, zun[z])) {
              t.reg[r++] = zreg[z];
              zi = z;
            }
          // One Z slab: its auxiliaries in a narrow box over its columns.
          if (r == 1) {
            const int ax = std::max(zun[zi].k0, k) & ~(halo - 1);
            t.ax = ax;
            wn = std::max(wn, std::min(zun[zi].k1, k + kSweepKW - 1) - ax + 1);
          }
          (r ? pml : bulk).push_back(t);
        }
  }
  if (!pml.empty() && !bulk.empty()) {
    std::vector<SweepTile> all;
    all.reserve(bulk.size() + pml.size());
    const size_t nb = bulk.size(), np = pml.size();
    for (size_t ib = 0, ip = 0; ib < nb || ip < np;) {
      if (ip < np && (ib >= nb || ip * (nb + 1) <= ib * (np + 1))) all.push_back(pml[ip++]);
      else all.push_back(bulk[ib++]);
    }
    pml.swap(all);
    bulk.clear();
  }
  // Narrow boxes must stay narrower than the full ones; else use those.
  wn = (wn + halo - 1) / halo * halo;
  if (wn > kSweepKW)
    for (SweepTile &t : pml) t.ax = -1;
  pl.wn = wn > kSweepKW ? 0 : wn;
  return pl;
}

template <typename T>
struct Engine : EngineBase {
  vgpu_problem p{};
  cudaStream_t s = nullptr;
  DevAlloc mem;
  Grid<T> g{};
  int n2p = 0;
  int64_t vol = 0;
  T *fields = nullptr;
  uint64_t *d_step = nullptr;
  // bulk
  Box be[3], bh[3], ube, ubh;
  // PML
  bool has_pml = false;
  PmlView<T> pv{};
  // Mur
  MurView mve{}, mvh{};
  unsigned mur_h_folded = 0;   // Mur faces whose normal H the H sweep updates (fold_mur_h)
  int64_t mur_total_e = 0, mur_total_h = 0;
  int64_t mur_max_e = 0, mur_max_h = 0;   // points of the largest item (launch grid x)
  // Debye
  DebyeItem *d_debye = nullptr;
  int n_debye = 0;
  int64_t debye_total = 0;
  double2 *d_J = nullptr, *d_dcoef = nullptr;
  T *d_lastE = nullptr;
  // SIBC
  int nsibc = 0;
  SibcSurf *d_surfs = nullptr;
  SibcModelDev *d_models = nullptr;
  double2 *d_q0 = nullptr, *d_q1 = nullptr, *d_q2 = nullptr, *d_zeta = nullptr;
  double *d_old = nullptr;
  uint8_t *d_adjA = nullptr, *d_adjB = nullptr;
  int64_t *d_zofs = nullptr;
  T *d_etan = nullptr;
  int64_t sibc_faces = 0;
  int64_t *d_tgt_index = nullptr, *d_tgt_start = nullptr;
  int *d_tgt_comp = nullptr;
  SibcOp<T> *d_ops = nullptr;
  int64_t ntgt = 0;
  // sources and plane waves
  std::vector<SrcLaunch> srcs;
  std::vector<PwLaunch<T>> pws;
  // ghost
  GhostView gv{};
  bool ghost_e = false, ghost_h = false;
  int ghost_threads = 0;
  // observers
  int *d_td_pts = nullptr, *d_fd_pts = nullptr;
  T *d_td = nullptr;
  double *d_stage = nullptr, *d_re = nullptr, *d_im = nullptr, *d_omega = nullptr;
  double2 *d_tw = nullptr;
  uint64_t nout = 0;
  uint64_t dft_folded = 0;   // output rows already folded into d_re/d_im
  // binary observers: device ring of 2 blocks x kChunk rows, pinned host copy
  int *d_bin_pts = nullptr;
  float *d_bin = nullptr, *h_bin = nullptr;
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_fill[2] = {}, ev_copy[2] = {};
  struct BinBlock {
    bool pending;
    uint64_t row0;
    uint32_t nrows;
  } bin_blk[2] = {};
  // TMA sweeps: tile lists and headers per launch, tensor maps per sweep,
  // full-volume UPML state.
  struct SweepLaunch {
    SweepTile *tiles = nullptr;
    std::vector<SweepTile> host;   // the same tiles, for grouped launches
    void *headers = nullptr;     // SweepHeader<T, PML>[ntiles]
    int ntiles = 0, grid = 0;
    uint32_t smem = 0;
    uint64_t bulk_points = 0, pml_points = 0;   // field points one launch updates
  };
  SweepLaunch sw_e[2], sw_h[2];   // [0] bulk kernel's tiles, [1] UPML kernel's tiles
  SweepMaps maps_e{}, maps_h{};
  PmlFull<T> pfe{}, pfh{};
  int pml_face[6] = {};
  int *d_err = nullptr;
  // FP64 sums of squares of E and H (k_energy), queued at every 64-step
  // boundary and at the problem's last step; energy_step is the step of the
  // latest one queued (0: none yet).
  double *d_energy = nullptr;
  uint64_t energy_step = 0;
  // Set-up work (uploads, clears, list preparation) runs on a stream of the
  // device's highest priority: with other engines stepping on the device,
  // its few small kernels start ahead of their queued sweep blocks.
  cudaStream_t ss = nullptr;
  // fused sweeps
  CoefIndex cie{}, cih{};
  // Merged side launches (k_side), decided at set-up by plan_side_merges.
  bool merge_e = false;      // the Debye cells and the plane wave's E corrections in one launch
  bool merge_obs = false;    // the plane wave's H corrections and the next step's samples in one launch
  bool need_sample = true;   // merge_obs: the current step's samples are still to be taken
  SideLaunch<T> side_e{}, side_h{};
  // step graphs (capture_graph)
  cudaGraphExec_t graphs[5] = {};
  uint64_t launches_per_step = 0;

  ~Engine() override
  {
    for (cudaGraphExec_t gx : graphs)
      if (gx) cudaGraphExecDestroy(gx);
    if (s) cudaStreamSynchronize(s);
    if (ss) cudaStreamSynchronize(ss);
    if (cs) cudaStreamSynchronize(cs);
    mem.free_all();
    if (h_bin) cudaFreeHost(h_bin);
    for (int q = 0; q < 2; q++) {
      if (ev_fill[q]) cudaEventDestroy(ev_fill[q]);
      if (ev_copy[q]) cudaEventDestroy(ev_copy[q]);
    }
    if (cs) cudaStreamDestroy(cs);
    if (ss) cudaStreamDestroy(ss);
    if (s) cudaStreamDestroy(s);
  }

  // This creation's pinned arena (null outside creation or when none could
  // be pinned) and the bytes of it already handed out.
  char *arena = nullptr;
  size_t arena_used = 0;
  static constexpr size_t kArenaMin = 256u << 10;   // smaller uploads go from pageable memory

  // A 256-byte-aligned slice of the arena for bytes about to be uploaded on
  // ss, or null if the arena is absent or full.
  char *arena_slice(size_t bytes)
  {
    if (!arena || bytes < kArenaMin || arena_used + bytes > PinnedArenas::kArena) return nullptr;
    char *a = arena + arena_used;
    arena_used += (bytes + 255) / 256 * 256;
    return a;
  }

  // bytes from host h to device d on the set-up stream.
  int put(void *d, const void *h, size_t bytes)
  {
    if (!bytes) return 0;
    const bool in_arena = arena && (const char *)h >= arena && (const char *)h < arena + PinnedArenas::kArena;
    if (!in_arena)
      if (char *a = arena_slice(bytes)) {
        host_copy(a, h, bytes);
        h = a;
      }
    CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ss));
    stats.h2d_bytes += bytes;
    return 0;
  }

  template <typename U>
  int upload(U **d, const U *h, size_t n)
  {
    if (mem.alloc(d, n)) return VGPU_ENOMEM;
    return put(*d, h, sizeof(U) * n);
  }

  // Copies n values into a device array of n + pad elements (zero tail), so
  // lanes of a tile that run into the row padding read valid memory.
  int upload_real(T **d, const double *h, size_t n, size_t pad = 0)
  {
    std::vector<T> tmp(n + pad ? n + pad : 1, (T)0);
    for (size_t q = 0; q < n; q++) tmp[q] = (T)h[q];
    if (mem.alloc(d, n + pad)) return VGPU_ENOMEM;
    return put(*d, tmp.data(), sizeof(T) * (n + pad));
  }

  // Host volume [n0][n1][n2] -> padded device volume.
  int upload_volume(T *d, const double *h)
  {
    std::vector<T> tmp((size_t)vol, (T)0);
    for (int i = 0; i < p.n[0]; i++)
      for (int j = 0; j < p.n[1]; j++) {
        const double *src = h + ((int64_t)i * p.n[1] + j) * p.n[2];
        T *dst = tmp.data() + (int64_t)i * g.s0 + (int64_t)j * g.s1;
        for (int k = 0; k < p.n[2]; k++) dst[k] = (T)src[k];
      }
    return put(d, tmp.data(), sizeof(T) * vol);
  }

  // With VGPU_TRACE set, create() prints the time of each set-up phase.
  struct PhaseClock {
    bool on = getenv("VGPU_TRACE") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    char buf[1024] = {};
    int len = 0;
    void mark(const char *name)
    {
      if (!on) return;
      auto now = std::chrono::steady_clock::now();
      double ms = std::chrono::duration<double, std::milli>(now - t).count();
      t = now;
      if (len < (int)sizeof buf - 64) len += snprintf(buf + len, sizeof buf - len, " %s %.2f", name, ms);
    }
    void print(int64_t vol) const
    {
      if (on) fprintf(stderr, "vgpu create (%lld cells, ms):%s\n", (long long)vol, buf);
    }
  };

  int create(const vgpu_problem *in)
  {
    PhaseClock pc;
    g_creating++;
    arena = pinned_arenas().take();
    arena_used = 0;
    int rc = create_phases(in, pc);
    // Every copy out of the arena has finished before it is handed back.
    if (ss) cudaStreamSynchronize(ss);
    pinned_arenas().give(arena);
    arena = nullptr;
    g_creating--;
    pclock = nullptr;
    pc.print(vol);
    return rc;
  }

  PhaseClock *pclock = nullptr;   // set while create() runs
  void mark(const char *name)
  {
    if (pclock) pclock->mark(name);
  }

  int create_phases(const vgpu_problem *in, PhaseClock &pc)
  {
    pclock = &pc;
    p = *in;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    {
      int least = 0, greatest = 0;
      CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      CK(cudaStreamCreateWithPriority(&ss, cudaStreamNonBlocking, greatest));
    }
    n2p = (p.n[2] + 31) / 32 * 32;
    g.n0 = p.n[0];
    g.n1 = p.n[1];
    g.n2 = p.n[2];
    g.s1 = n2p;
    g.s0 = (int64_t)p.n[1] * n2p;
    vol = (int64_t)p.n[0] * g.s0;
    if (mem.alloc(&fields, (size_t)vol * 6)) return VGPU_ENOMEM;
    CK(cudaMemsetAsync(fields, 0, sizeof(T) * vol * 6, ss));
    for (int c = 0; c < 6; c++) g.F[c] = fields + (int64_t)c * vol;
    pc.mark("fields");
    // Coefficients: a one-byte index and a table where the mesh allows it
    // (at most 256 distinct tuples), else the full volumes.
    if (int rc = setup_coef_index()) return rc;
    g.cidx[0] = cie.idx;
    g.ctab[0] = (const T *)cie.table;
    g.cidx[1] = cih.idx;
    g.ctab[1] = (const T *)cih.table;
    for (int grp = 0; grp < 2; grp++) {
      if ((grp == 0 ? cie : cih).idx) continue;
      const int q0 = grp == 0 ? 0 : 6, nq = grp == 0 ? 6 : 3;
      T *coef = nullptr;
      if (mem.alloc(&coef, (size_t)vol * nq)) return VGPU_ENOMEM;
      for (int q = 0; q < nq; q++) {
        if (int rc = upload_volume(coef + (int64_t)q * vol, p.coef[q0 + q])) return rc;
        g.cf[q0 + q] = coef + (int64_t)q * vol;
      }
    }
    for (int a = 0; a < 3; a++) {
      T *d;
      if (int rc = upload_real(&d, p.ide[a], p.n[a], 64)) return rc;
      g.ide[a] = d;
      if (int rc = upload_real(&d, p.idh[a], p.n[a], 64)) return rc;
      g.idh[a] = d;
    }
    if (mem.alloc(&d_step, 1)) return VGPU_ENOMEM;
    CK(cudaMemsetAsync(d_step, 0, sizeof(uint64_t), ss));
    pc.mark(p.num_tags > 0 && p.tag_coef ? "coef-from-tags" : "coef");

    // Bulk limits.
    for (int c = 0; c < 3; c++) {
      be[c] = box_from(p.gfilim[c]);
      bh[c] = box_from(p.gfilim[3 + c]);
    }
    ube = unite(be);
    ubh = unite(bh);

    if (int rc = setup_pml()) return rc;
    mur_h_folded = fold_mur_h(p, bh);
    ubh = unite(bh);
    if (int rc = setup_mur()) return rc;
    if (int rc = setup_debye()) return rc;
    if (int rc = setup_sibc()) return rc;
    if (int rc = setup_sources()) return rc;
    pc.mark("pml-mur-debye-sibc-src");
    if (int rc = setup_planewaves()) return rc;
    pc.mark("tfsf");
    setup_ghost();
    if (int rc = setup_observers()) return rc;
    pc.mark("observers");
    if (int rc = setup_sweeps()) return rc;
    plan_side_merges();
    // The read-back stage is pinned once per process, by the first engine
    // created, so no read pays for it.
    if (int rc = pinned_stage().ensure_locked()) return rc;
    CK(cudaStreamSynchronize(ss));
    CK(cudaGetLastError());
    pc.mark("sweeps");
    stats.device_bytes = mem.bytes;
    int rc = capture_graph();
    pc.mark("graph");
    return rc;
  }


  int setup_pml()
  {
    pv.nreg = 0;
    for (int r = 0; r < 6; r++) {
      if (!p.pml_present[r]) continue;
      int q = pv.nreg++;
      pml_face[q] = r;
      Box bb[6];
      for (int f = 0; f < 6; f++) bb[f] = box_from(p.pml_flim[r][f]);
      for (int f = 0; f < 6; f++) pv.lim[q][f] = bb[f];
    }
    has_pml = pv.nreg > 0;
    if (!has_pml) return 0;
    for (int a = 0; a < 3; a++) {
      T *d;
      if (int rc = upload_real(&d, p.pml_ad[a], p.n[a], 64)) return rc; pv.ad[a] = d;
      if (int rc = upload_real(&d, p.pml_bd[a], p.n[a], 64)) return rc; pv.bd[a] = d;
      if (int rc = upload_real(&d, p.pml_ah[a], p.n[a], 64)) return rc; pv.ah[a] = d;
      if (int rc = upload_real(&d, p.pml_bh[a], p.n[a], 64)) return rc; pv.bh[a] = d;
      if (int rc = upload_real(&d, p.pml_ibd[a], p.n[a], 64)) return rc; pv.ibd[a] = d;
      if (int rc = upload_real(&d, p.pml_ibh[a], p.n[a], 64)) return rc; pv.ibh[a] = d;
    }
    return 0;
  }

  int setup_mur()
  {
    mve.nitems = mvh.nitems = 0;
    mur_total_e = mur_total_h = 0;
    for (int f = 0; f < 6; f++) {
      mve.zeta[f] = mvh.zeta[f] = p.mur_zeta[f];
      if (!p.mur_present[f]) continue;
      int a = f / 2;
      int dir = (f % 2 == 0) ? +1 : -1;
      int comps[2];
      if (a == 0) { comps[0] = EY; comps[1] = EZ; }
      else if (a == 1) { comps[0] = EX; comps[1] = EZ; }
      else { comps[0] = EY; comps[1] = EX; }
      for (int cc = 0; cc < 2; cc++) {
        Box b = box_from(p.mur_flim[f][comps[cc]]);
        if (b.empty()) continue;
        MurItem &m = mve.it[mve.nitems++];
        m.b = b; m.c = comps[cc]; m.axis = a; m.dir = dir; m.face = f; m.first = mur_total_e;
        mur_total_e += b.count();
        mur_max_e = std::max(mur_max_e, b.count());
      }
      Box b = box_from(p.mur_flim[f][HX + a]);
      if (!b.empty() && !(mur_h_folded >> f & 1u)) {
        MurItem &m = mvh.it[mvh.nitems++];
        m.b = b; m.c = HX + a; m.axis = a; m.dir = 0; m.face = f; m.first = mur_total_h;
        mur_total_h += b.count();
        mur_max_h = std::max(mur_max_h, b.count());
      }
    }
    if (std::max(mur_max_e, mur_max_h) >= ((int64_t)1 << 31))
      return set_err(VGPU_EINVAL, "a Mur face of %lld points exceeds the engine's limit",
                     (long long)std::max(mur_max_e, mur_max_h));
    return 0;
  }

  int setup_debye()
  {
    std::vector<DebyeItem> items;
    std::vector<double2> coefs;
    int64_t total = 0, jtot = 0, etot = 0;
    for (int b = 0; b < p.num_debye; b++) {
      const vgpu_debye &d = p.debye[b];
      int ofs = (int)coefs.size();
      for (int q = 0; q < d.num_poles; q++) coefs.push_back(make_double2(d.dalpha[2 * q], d.dalpha[2 * q + 1]));
      for (int q = 0; q < d.num_poles; q++) coefs.push_back(make_double2(d.dbeta[2 * q], d.dbeta[2 * q + 1]));
      for (int c = 0; c < 3; c++) {
        Box bx = box_from(d.flim[c]);
        if (bx.empty()) continue;
        DebyeItem it{};
        it.b = bx; it.c = c; it.np = d.num_poles; it.first = total; it.jofs = jtot; it.eofs = etot; it.coef_ofs = ofs;
        if (bx.count() >= ((int64_t)1 << 31))
          return set_err(VGPU_EINVAL, "a Debye block of %lld cells exceeds the engine's limit", (long long)bx.count());
        items.push_back(it);
        total += bx.count();
        jtot += bx.count() * d.num_poles;
        etot += bx.count();
      }
    }
    n_debye = (int)items.size();
    debye_total = total;
    if (!n_debye) return 0;
    if (int rc = upload(&d_debye, items.data(), items.size())) return rc;
    if (int rc = upload(&d_dcoef, coefs.data(), coefs.size())) return rc;
    if (mem.alloc(&d_J, jtot) || mem.alloc(&d_lastE, etot)) return VGPU_ENOMEM;
    CK(cudaMemsetAsync(d_J, 0, sizeof(double2) * (jtot ? jtot : 1), ss));
    CK(cudaMemsetAsync(d_lastE, 0, sizeof(T) * (etot ? etot : 1), ss));
    return 0;
  }

  int setup_sibc()
  {
    nsibc = p.num_sibc;
    if (!nsibc) return 0;
    std::vector<SibcModelDev> models(p.num_sibc_models);
    int total_poles = 0;
    for (int m = 0; m < p.num_sibc_models; m++) {
      const vgpu_sibc_model &sm = p.sibc_models[m];
      models[m].poles = 0;
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
          models[m].np[a][b] = sm.num_poles[a][b];
          models[m].off[a][b] = sm.pole_offset[a][b];
          models[m].asymp[a][b] = sm.asymp[a][b];
          models[m].poles += sm.num_poles[a][b];
          total_poles = std::max(total_poles, sm.pole_offset[a][b] + sm.num_poles[a][b]);
        }
    }
    std::vector<double2> q0(total_poles + 1), q1(total_poles + 1), q2(total_poles + 1);
    if (p.num_sibc_models) {
      const vgpu_sibc_model &sm = p.sibc_models[0];
      for (int r = 0; r < total_poles; r++) {
        q0[r] = make_double2(sm.q0[2 * r], sm.q0[2 * r + 1]);
        q1[r] = make_double2(sm.q1[2 * r], sm.q1[2 * r + 1]);
        q2[r] = make_double2(sm.q2[2 * r], sm.q2[2 * r + 1]);
      }
    }
    std::vector<SibcSurf> surfs(nsibc);
    std::vector<int64_t> zofs(nsibc + 1), base(nsibc + 1);
    std::vector<uint8_t> adjA, adjB;
    int64_t faces = 0, z = 0;
    for (int q = 0; q < nsibc; q++) {
      const vgpu_sibc_surface &sf = p.sibc[q];
      SibcSurf &o = surfs[q];
      o.g = Box{ sf.gbbox[0], sf.gbbox[1] - 1, sf.gbbox[2], sf.gbbox[3] - 1, sf.gbbox[4], sf.gbbox[5] - 1 };
      o.normal = sf.normal;
      o.model = sf.model;
      o.first = faces;
      memcpy(o.A, sf.A, sizeof o.A);
      memcpy(o.B, sf.B, sizeof o.B);
      int64_t nf = o.g.count();
      if (nf >= ((int64_t)1 << 31))
        return set_err(VGPU_EINVAL, "an SIBC surface of %lld faces exceeds the engine's limit", (long long)nf);
      base[q] = faces;
      zofs[q] = z;
      adjA.insert(adjA.end(), sf.adjA, sf.adjA + 4 * nf);
      adjB.insert(adjB.end(), sf.adjB, sf.adjB + 4 * nf);
      faces += nf;
      z += nf * models[sf.model].poles;
    }
    sibc_faces = faces;
    if (upload(&d_surfs, surfs.data(), surfs.size()) || upload(&d_models, models.data(), models.size()) ||
        upload(&d_q0, q0.data(), q0.size()) || upload(&d_q1, q1.data(), q1.size()) ||
        upload(&d_q2, q2.data(), q2.size()) || upload(&d_adjA, adjA.data(), adjA.size()) ||
        upload(&d_adjB, adjB.data(), adjB.size()) || upload(&d_zofs, zofs.data(), zofs.size()))
      return VGPU_ENOMEM;
    if (mem.alloc(&d_zeta, z) || mem.alloc(&d_old, faces * 16) || mem.alloc(&d_etan, faces * 4)) return VGPU_ENOMEM;
    CK(cudaMemsetAsync(d_zeta, 0, sizeof(double2) * (z ? z : 1), ss));
    CK(cudaMemsetAsync(d_old, 0, sizeof(double) * (faces ? faces * 16 : 1), ss));
    CK(cudaMemsetAsync(d_etan, 0, sizeof(T) * (faces ? faces * 4 : 1), ss));
    if (faces * 4 > INT32_MAX) return set_err(VGPU_EINVAL, "%lld SIBC faces exceed the engine's limit", (long long)faces);
    // Magnetic correction targets (ops arrive sorted by target).
    std::vector<int64_t> tidx, tstart;
    std::vector<int> tcomp;
    std::vector<SibcOp<T>> ops((size_t)p.num_sibc_hops + 1);
    for (int64_t h = 0; h < p.num_sibc_hops; h++) {
      const vgpu_sibc_hop &o = p.sibc_hops[h];
      int i = (int)(o.index / ((int64_t)p.n[1] * p.n[2]));
      int j = (int)((o.index / p.n[2]) % p.n[1]);
      int k = (int)(o.index % p.n[2]);
      int64_t dx = (int64_t)i * g.s0 + (int64_t)j * g.s1 + k;
      if (h == 0 || o.index != p.sibc_hops[h - 1].index || o.comp != p.sibc_hops[h - 1].comp) {
        tidx.push_back(dx);
        tcomp.push_back(o.comp);
        tstart.push_back(h);
      }
      SibcOp<T> &d = ops[h];
      d.kind = o.kind;
      d.c = (T)o.c; d.d1 = (T)o.d1; d.d2 = (T)o.d2; d.n1 = (T)o.n1; d.n2 = (T)o.n2;
      d.e1 = (int32_t)(4 * (base[o.s1] + o.f1) + o.slot1);
      d.e2 = (int32_t)(4 * (base[o.s2] + o.f2) + o.slot2);
    }
    tstart.push_back(p.num_sibc_hops);
    ntgt = (int64_t)tidx.size();
    if (upload(&d_tgt_index, tidx.data(), tidx.size()) || upload(&d_tgt_comp, tcomp.data(), tcomp.size()) ||
        upload(&d_tgt_start, tstart.data(), tstart.size()) || upload(&d_ops, ops.data(), ops.size()))
      return VGPU_ENOMEM;
    return 0;
  }

  int setup_sources()
  {
    for (int q = 0; q < p.num_sources; q++) {
      const vgpu_source &src = p.sources[q];
      SrcLaunch l{};
      l.b = box_from(src.flim);
      l.c = src.field;
      l.kind = src.kind;
      l.soft = src.soft;
      T *d;
      if (int rc = upload_real(&d, src.values, p.num_steps)) return rc;
      l.values = d;
      if (!l.b.empty()) srcs.push_back(l);
    }
    return 0;
  }

  int setup_planewaves()
  {
    static const int face_order[6] = { 2, 3, 4, 5, 0, 1 };  // YLO YHI ZLO ZHI XLO XHI
    // (component, incident component, sign) per face for E and for H (src/planewave.c:576-1007).
    static const int ecorr[6][2][3] = {
      { { EY, HZ, +1 }, { EZ, HY, -1 } },  // XLO
      { { EY, HZ, -1 }, { EZ, HY, +1 } },  // XHI
      { { EX, HZ, -1 }, { EZ, HX, +1 } },  // YLO
      { { EX, HZ, +1 }, { EZ, HX, -1 } },  // YHI
      { { EX, HY, +1 }, { EY, HX, -1 } },  // ZLO
      { { EX, HY, -1 }, { EY, HX, +1 } },  // ZHI
    };
    static const int hcorr[6][2][3] = {
      { { HZ, EY, +1 }, { HY, EZ, -1 } },  // XLO
      { { HZ, EY, -1 }, { HY, EZ, +1 } },  // XHI
      { { HZ, EX, -1 }, { HX, EZ, +1 } },  // YLO
      { { HZ, EX, +1 }, { HX, EZ, -1 } },  // YHI
      { { HY, EX, +1 }, { HX, EY, -1 } },  // ZLO
      { { HY, EX, -1 }, { HX, EY, +1 } },  // ZHI
    };
    std::vector<const double *> pos;
    double *pn[3], *ph[3];
    if (p.num_planewaves) {
      for (int a = 0; a < 3; a++) {
        if (upload(&pn[a], p.pos_node[a], p.n[a]) || upload(&ph[a], p.pos_half[a], p.n[a])) return VGPU_ENOMEM;
      }
    }
    for (int q = 0; q < p.num_planewaves; q++) {
      const vgpu_planewave &w = p.planewaves[q];
      PwLaunch<T> L{};
      PwView<T> &v = L.pv;
      v.use_aux = w.use_aux_grid;
      const vgpu_waveform &wf = p.waveforms[w.waveform];
      v.wf.type = wf.type; v.wf.table_size = wf.table_size; v.wf.size = wf.size; v.wf.delay = wf.delay;
      v.wf.width = wf.width; v.wf.frequency = wf.frequency; v.wf.table = nullptr;
      if (wf.type == VGPU_WF_EXTERNAL) {
        double *dt_;
        if (upload(&dt_, wf.table, (size_t)wf.table_size * 3)) return VGPU_ENOMEM;
        v.wf.table = dt_;
      }
      v.delay = w.delay;
      v.phase_velocity = w.phase_velocity;
      for (int a = 0; a < 3; a++) {
        v.kinc[a] = w.kinc[a]; v.r0[a] = w.r0[a]; v.ijk0[a] = w.ijk0[a];
        v.pos_node[a] = pn[a]; v.pos_half[a] = ph[a];
      }
      for (int c = 0; c < 6; c++) v.finc[c] = w.finc[c];
      if (w.use_aux_grid) {
        v.nx = w.aux_nx;
        v.xb = w.aux_xb;
        v.beta = (T)w.aux_beta;
        v.gamma = (T)w.aux_gamma;
        double mu0 = 4.0 * (4.0 * atan(1.0)) * 1e-7;
        v.eta0 = (T)sqrt(mu0 / (1.0 / (mu0 * 299792458.0 * 299792458.0)));
        if (mem.alloc(&v.Eyi, w.aux_nx + 2) || mem.alloc(&v.Hzi, w.aux_nx + 2) || mem.alloc(&v.PPyi, w.aux_npml) ||
            mem.alloc(&v.Pyi, w.aux_npml) || mem.alloc(&v.Bzi, w.aux_npml))
          return VGPU_ENOMEM;
        CK(cudaMemsetAsync(v.Eyi, 0, sizeof(T) * (w.aux_nx + 2), ss));
        CK(cudaMemsetAsync(v.Hzi, 0, sizeof(T) * (w.aux_nx + 2), ss));
        CK(cudaMemsetAsync(v.PPyi, 0, sizeof(T) * w.aux_npml, ss));
        CK(cudaMemsetAsync(v.Pyi, 0, sizeof(T) * w.aux_npml, ss));
        CK(cudaMemsetAsync(v.Bzi, 0, sizeof(T) * w.aux_npml, ss));
        T *d;
        if (upload_real(&d, w.aux_adx, w.aux_npml)) return VGPU_ENOMEM; v.adx = d;
        if (upload_real(&d, w.aux_bdx, w.aux_npml)) return VGPU_ENOMEM; v.bdx = d;
        if (upload_real(&d, w.aux_ahx, w.aux_npml)) return VGPU_ENOMEM; v.ahx = d;
        if (upload_real(&d, w.aux_bhx, w.aux_npml)) return VGPU_ENOMEM; v.bhx = d;
        if (upload_real(&d, w.aux_source, p.num_steps)) return VGPU_ENOMEM; v.source = d;
      }
      L.te.n = L.th.n = 0;
      for (int o = 0; o < 6; o++) {
        int f = face_order[o];
        if (!w.active[f]) continue;
        int a = f / 2;
        bool lo = f % 2 == 0;
        for (int e = 0; e < 2; e++) {
          Box b = box_from(w.flim[f][ecorr[f][e][0]]);
          if (!b.empty()) {
            TfsfItem &it = L.te.it[L.te.n++];
            it.b = b; it.c = ecorr[f][e][0]; it.inc = ecorr[f][e][1]; it.sign = ecorr[f][e][2];
            it.axis = a; it.shift = lo ? -1 : 0; it.first = L.total_e;
            L.total_e += b.count();
          }
          b = box_from(w.flim[f][hcorr[f][e][0]]);
          if (!b.empty()) {
            TfsfItem &it = L.th.it[L.th.n++];
            it.b = b; it.c = hcorr[f][e][0]; it.inc = hcorr[f][e][1]; it.sign = hcorr[f][e][2];
            it.axis = a; it.shift = lo ? +1 : 0; it.first = L.total_h;
            L.total_h += b.count();
          }
        }
      }
      if (int rc = build_tfsf_list(L, true)) return rc;
      if (int rc = build_tfsf_list(L, false)) return rc;
      pws.push_back(L);
    }
    return 0;
  }

  // The point list of one plane wave's E or H corrections (TfsfList):
  // entries in the reference's face order, grouped by point, with the
  // step-independent part of each incident field precomputed on the device.
  int build_tfsf_list(PwLaunch<T> &L, bool efield)
  {
    const TfsfView &tv = efield ? L.te : L.th;
    TfsfList<T> &tl = efield ? L.le : L.lh;
    // A point belongs to the first item (in face order) that holds it; the
    // later items of the same component that hold it follow it in its run.
    // Each item's points, in its i, j, k order, are cut into ranges that are
    // enumerated on separate host threads and joined in item and range order.
    struct Part {
      int q;                                 // item
      int64_t lo, hi;                        // range of the item's points
      std::vector<int64_t> sx, mx;           // field indices of single- and multi-entry points
      std::vector<uint8_t> sq, mq;           // their items
      std::vector<int> mstart;               // run starts within the multi entries
    };
    std::vector<Part> parts;
    {
      int64_t total = 0;
      for (int q = 0; q < tv.n; q++) total += tv.it[q].b.count();
      const int64_t chunk = std::max<int64_t>(4096, total / (2 * host_threads()) + 1);
      for (int q = 0; q < tv.n; q++)
        for (int64_t lo = 0, n = tv.it[q].b.count(); lo < n; lo += chunk) {
          parts.emplace_back();
          parts.back().q = q;
          parts.back().lo = lo;
          parts.back().hi = std::min(n, lo + chunk);
        }
    }
    const int nparts = (int)parts.size();
    // An entry is sent as its field index and item; the device fills in the
    // rest (k_tfsf_prepare), from the arrays the sweeps read.
    auto make = [&](int q, int i, int j, int k, std::vector<int64_t> &xs, std::vector<uint8_t> &qs) {
      xs.push_back((int64_t)i * g.s0 + (int64_t)j * g.s1 + k);
      qs.push_back((uint8_t)q);
    };
    auto enumerate = [&](int w) {
      Part &pt = parts[w];
      const int q = pt.q;
      const TfsfItem &it = tv.it[q];
      // Other items of the component that meet this one.
      int others[12], no = 0;
      for (int e = 0; e < tv.n; e++)
        if (e != q && tv.it[e].c == it.c && boxes_meet(tv.it[e].b, it.b)) others[no++] = e;
      pt.sx.reserve(pt.hi - pt.lo);
      pt.sq.reserve(pt.hi - pt.lo);
      const int64_t njk = (int64_t)it.b.nj() * it.b.nk();
      int i = it.b.i0 + (int)(pt.lo / njk), j = it.b.j0 + (int)(pt.lo % njk / it.b.nk()),
          k = it.b.k0 + (int)(pt.lo % it.b.nk());
      for (int64_t x = pt.lo; x < pt.hi; x++) {
        if (x > pt.lo && ++k > it.b.k1) {
          k = it.b.k0;
          if (++j > it.b.j1) {
            j = it.b.j0;
            i++;
          }
        }
        bool owned = true, followers = false;
        for (int o = 0; o < no && owned; o++) {
          if (!tv.it[others[o]].b.contains(i, j, k)) continue;
          if (others[o] < q) owned = false;
          else followers = true;
        }
        if (!owned) continue;
        if (!followers) {
          make(q, i, j, k, pt.sx, pt.sq);
          continue;
        }
        pt.mstart.push_back((int)pt.mx.size());
        make(q, i, j, k, pt.mx, pt.mq);
        for (int o = 0; o < no; o++)
          if (others[o] > q && tv.it[others[o]].b.contains(i, j, k)) make(others[o], i, j, k, pt.mx, pt.mq);
      }
    };
    mark(efield ? "tfsf-e-start" : "tfsf-h-start");
    HostPool::get().run(nparts, enumerate);
    mark("enumerate");
    // Points of one entry first, then the multi-entry points' runs.
    size_t ns = 0, nm = 0;
    for (const Part &pt : parts) {
      ns += pt.sx.size();
      nm += pt.mx.size();
    }
    const size_t ne = ns + nm;
    // Each part's runs go to their final offsets, one host thread per part.
    std::vector<size_t> soff(nparts + 1, 0), moff(nparts + 1, ns);
    for (int q = 0; q < nparts; q++) {
      soff[q + 1] = soff[q] + parts[q].sx.size();
      moff[q + 1] = moff[q] + parts[q].mx.size();
    }
    // The merged lists are written where they are sent from: the
    // creation's pinned arena when it has room.
    std::vector<int64_t> xs_v;
    std::vector<uint8_t> qs_v;
    std::vector<int> mstart;
    int64_t *xs = (int64_t *)arena_slice(sizeof(int64_t) * ne);
    uint8_t *qs = (uint8_t *)arena_slice(ne);
    if (!xs) {
      xs_v.resize(ne);
      xs = xs_v.data();
    }
    if (!qs) {
      qs_v.resize(ne);
      qs = qs_v.data();
    }
    {
      auto place = [&](int q) {
        const Part &pt = parts[q];
        std::copy(pt.sx.begin(), pt.sx.end(), xs + soff[q]);
        std::copy(pt.sq.begin(), pt.sq.end(), qs + soff[q]);
        std::copy(pt.mx.begin(), pt.mx.end(), xs + moff[q]);
        std::copy(pt.mq.begin(), pt.mq.end(), qs + moff[q]);
      };
      HostPool::get().run(nparts, place);
    }
    for (int q = 0; q < nparts; q++)
      for (int m : parts[q].mstart) mstart.push_back((int)moff[q] + m);
    mstart.push_back((int)ne);
    mark("merge");
    tl.nentries = (int64_t)ne;
    tl.nsingle = (int)ns;
    tl.nmulti = (int)mstart.size() - 1;
    if (!ne) return 0;
    TfsfEntry<T> *de;
    int64_t *dx;
    uint8_t *dq;
    int *dm;
    if (mem.alloc(&de, ne) || upload(&dx, xs, ne) || upload(&dq, qs, ne) || upload(&dm, mstart.data(), mstart.size()))
      return VGPU_ENOMEM;
    tl.ent = de;
    tl.seed_x = dx;
    tl.seed_q = dq;
    tl.mstart = dm;
    mark("upload");
    k_tfsf_prepare<T><<<blocks_for(ne, 128), 128, 0, ss>>>(g, L.pv, tv, tl, efield ? 1 : 0);
    CK(cudaGetLastError());
    mark("prepare");
    return 0;
  }

  // Distinct coefficient tuples per cell: (alpha, beta) x 3 for E and
  // gamma x 3 for H.  Up to 256 tuples compress to one byte per cell.  The
  // i planes are split among host threads; each numbers the tuples it meets,
  // and the tables merge in plane order, so the numbering does not depend on
  // the thread count.
  int build_index(int first, int count, CoefIndex &out)
  {
    out = CoefIndex{};
    struct Key {
      T v[6];
      bool operator<(const Key &o) const { return memcmp(v, o.v, sizeof v) < 0; }
    };
    const int n0 = p.n[0];
    const int nthr = std::max(1, std::min<int>(host_threads(), n0));
    // Written where it is sent from: the creation's pinned arena when it has
    // room (the row padding past n2 is never read).
    std::vector<uint8_t> idx_v;
    uint8_t *idx = (uint8_t *)arena_slice((size_t)vol);
    if (!idx) {
      idx_v.assign((size_t)vol, 0);
      idx = idx_v.data();
    }
    struct Part {
      std::vector<Key> keys;   // local tuples in first-seen order
      bool overflow = false;
      int bad_tag = 0;         // a tag past the problem's table, if met
    };
    std::vector<Part> parts(nthr);
    // With medium tags a cell's tuple follows from its components' tag bytes
    // (three per cell for E or H) instead of its doubles.  The cells are
    // walked in the same order and each tuple is keyed by its values, so the
    // index and the table are the ones the scan of the volumes gives.
    // Volume q of coef[] is the alpha (q < 3), beta (q < 6) or gamma of the
    // component whose tags are coef_tag[q < 3 ? q : q - 3].
    bool tagged = p.num_tags > 0 && p.num_tags <= 255 && p.tag_coef;
    for (int c = 0; c < count && tagged; c++) tagged = p.coef_tag[first + c < 3 ? first + c : first + c - 3] != nullptr;
    auto work_tags = [&](int w) {
      const int i0 = (int)((int64_t)n0 * w / nthr), i1 = (int)((int64_t)n0 * (w + 1) / nthr);
      Part &pt = parts[w];
      std::map<Key, int> seen;
      const int tv0 = first < 3 ? 0 : 3;     // the three tag volumes: tv0 .. tv0 + 2
      const uint8_t *tg[3];
      for (int c = 0; c < 3; c++) tg[c] = p.coef_tag[tv0 + c];
      int vol_tag[6], vol_slot[6];
      for (int c = 0; c < count; c++) {
        const int q = first + c;
        vol_tag[c] = (q < 3 ? q : q - 3) - tv0;
        vol_slot[c] = q < 3 ? 0 : q < 6 ? 1 : 2;
      }
      int last = -1;
      uint8_t lastt[3] = {};
      int64_t prev_hrow = -1;
      const uint8_t *prev_irow = nullptr;
      for (int i = i0; i < i1 && !pt.overflow; i++)
        for (int j = 0; j < p.n[1]; j++) {
          const int64_t hrow = ((int64_t)i * p.n[1] + j) * p.n[2];
          uint8_t *irow = idx + (int64_t)i * g.s0 + (int64_t)j * g.s1;
          if (prev_irow && memcmp(tg[0] + hrow, tg[0] + prev_hrow, (size_t)p.n[2]) == 0 &&
              memcmp(tg[1] + hrow, tg[1] + prev_hrow, (size_t)p.n[2]) == 0 &&
              memcmp(tg[2] + hrow, tg[2] + prev_hrow, (size_t)p.n[2]) == 0) {
            memcpy(irow, prev_irow, (size_t)p.n[2]);
            prev_hrow = hrow;
            prev_irow = irow;
            continue;
          }
          prev_hrow = hrow;
          prev_irow = irow;
          for (int k = 0; k < p.n[2]; k++) {
            const uint8_t t[3] = { tg[0][hrow + k], tg[1][hrow + k], tg[2][hrow + k] };
            if (last >= 0 && t[0] == lastt[0] && t[1] == lastt[1] && t[2] == lastt[2]) {
              irow[k] = (uint8_t)last;
              continue;
            }
            Key key{};
            for (int c = 0; c < count; c++) {
              const uint8_t tc = t[vol_tag[c]];
              if (tc > p.num_tags) {
                pt.bad_tag = tc;
                return;
              }
              key.v[c] = tc ? (T)p.tag_coef[(tc - 1) * 3 + vol_slot[c]] : (T)0.0;
            }
            int q = -1;
            auto it = seen.find(key);
            if (it != seen.end()) q = it->second;
            if (q < 0) {
              if (seen.size() == 256) {
                pt.overflow = true;
                return;
              }
              q = (int)seen.size();
              seen.emplace(key, q);
              pt.keys.push_back(key);
            }
            last = q;
            memcpy(lastt, t, sizeof t);
            irow[k] = (uint8_t)q;
          }
        }
    };
    auto work = [&](int w) {
      const int i0 = (int)((int64_t)n0 * w / nthr), i1 = (int)((int64_t)n0 * (w + 1) / nthr);
      Part &pt = parts[w];
      std::map<Key, int> seen;
      int last = -1;
      uint64_t lastraw[6] = {};   // bit patterns of the previous cell's doubles
      const double *src[6];
      for (int c = 0; c < count; c++) src[c] = p.coef[first + c];
      int64_t prev_hrow = -1;
      const uint8_t *prev_irow = nullptr;
      for (int i = i0; i < i1 && !pt.overflow; i++)
        for (int j = 0; j < p.n[1]; j++) {
          const int64_t hrow = ((int64_t)i * p.n[1] + j) * p.n[2];
          uint8_t *irow = idx + (int64_t)i * g.s0 + (int64_t)j * g.s1;
          // A row whose doubles equal the row before (the common case):
          // the same tuples, compared and copied a row at a time.
          if (prev_irow) {
            bool same = true;
            for (int c = 0; c < count && same; c++)
              same = memcmp(src[c] + hrow, src[c] + prev_hrow, sizeof(double) * (size_t)p.n[2]) == 0;
            if (same) {
              memcpy(irow, prev_irow, (size_t)p.n[2]);
              prev_hrow = hrow;
              prev_irow = irow;
              continue;
            }
          }
          prev_hrow = hrow;
          prev_irow = irow;
          for (int k = 0; k < p.n[2]; k++) {
            // Same doubles as the previous cell (the common case): same tuple.
            uint64_t raw[6];
            bool same = last >= 0;
            for (int c = 0; c < count; c++) {
              memcpy(&raw[c], src[c] + hrow + k, sizeof(double));
              same = same && raw[c] == lastraw[c];
            }
            if (same) {
              irow[k] = (uint8_t)last;
              continue;
            }
            Key key{};
            for (int c = 0; c < count; c++) key.v[c] = (T)src[c][hrow + k];
            int q = -1;
            auto it = seen.find(key);
            if (it != seen.end()) q = it->second;
            if (q < 0) {
              if (seen.size() == 256) {
                pt.overflow = true;
                return;
              }
              q = (int)seen.size();
              seen.emplace(key, q);
              pt.keys.push_back(key);
            }
            last = q;
            memcpy(lastraw, raw, sizeof raw);
            irow[k] = (uint8_t)q;
          }
        }
    };
    if (tagged)
      HostPool::get().run(nthr, work_tags);
    else
      HostPool::get().run(nthr, work);
    for (const Part &pt : parts)
      if (pt.bad_tag)
        return set_err(VGPU_EINVAL, "medium tag %d is past the problem's %d tags", pt.bad_tag, (int)p.num_tags);
    // Merge: global numbers in plane order, then renumber each part's planes.
    std::map<Key, int> global;
    std::vector<T> table;
    std::vector<std::array<uint8_t, 256>> remap(nthr);
    std::vector<char> ident(nthr, 1);
    for (int w = 0; w < nthr; w++) {
      if (parts[w].overflow) return 0;  // too many: keep the full volumes
      remap[w].fill(0);
      for (size_t q = 0; q < parts[w].keys.size(); q++) {
        const Key &key = parts[w].keys[q];
        auto it = global.find(key);
        if (it == global.end()) {
          if (global.size() == 256) return 0;
          it = global.emplace(key, (int)global.size()).first;
          for (int c = 0; c < count; c++) table.push_back(key.v[c]);
        }
        remap[w][q] = (uint8_t)it->second;
        ident[w] = ident[w] && it->second == (int)q;
      }
    }
    // Each part renumbers its own planes, on its own thread.
    HostPool::get().run(nthr, [&](int w) {
      if (ident[w]) return;
      const int i0 = (int)((int64_t)n0 * w / nthr), i1 = (int)((int64_t)n0 * (w + 1) / nthr);
      const uint8_t *rm = remap[w].data();
      for (int64_t x = (int64_t)i0 * g.s0; x < (int64_t)i1 * g.s0; x++) idx[x] = rm[idx[x]];
    });
    uint8_t *d_idx;
    T *d_tab;
    if (upload(&d_idx, idx, (size_t)vol) || upload(&d_tab, table.data(), table.size())) return VGPU_ENOMEM;
    out.idx = d_idx;
    out.table = d_tab;
    out.ntab = (int)global.size();
    return 0;
  }


  // ---- TMA sweeps ------------------------------------------------------

  static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
  {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!fn) {
      void *ptr = nullptr;
      cudaDriverEntryPointQueryResult q{};
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
          q == cudaDriverEntryPointSuccess)
        fn = (PFN_cuTensorMapEncodeTiled_v12000)ptr;
    }
    return fn;
  }

  // A 3-D map over one [n0][n1][n2p] volume with box (bx, by, 1).  Its k
  // extent is n2, not the padded row: columns past the grid read as zero
  // without touching memory.
  int make_map(CUtensorMap *m, const void *base, CUtensorMapDataType dt, int esize, int bx, int by)
  {
    auto fn = encode_fn();
    if (!fn) return set_err(VGPU_ECUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t dims[3] = { (cuuint64_t)p.n[2], (cuuint64_t)p.n[1], (cuuint64_t)p.n[0] };
    cuuint64_t strides[2] = { (cuuint64_t)n2p * esize, (cuuint64_t)n2p * p.n[1] * esize };
    cuuint32_t box[3] = { (cuuint32_t)bx, (cuuint32_t)by, 1 };
    cuuint32_t es[3] = { 1, 1, 1 };
    CUresult r = fn(m, dt, 3, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_64B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(VGPU_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
  }

  // Maps of one sweep: own = the updated components, oth = the curl's.
  // Curl boxes carry a 16-byte halo column; the others are one tile row.
  int make_sweep_maps(SweepMaps &m, bool esweep)
  {
    const int jh = kSweepJH, wc = kSweepKW + 16 / (int)sizeof(T), w = kSweepKW;
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const int e = (int)sizeof(T);
    for (int c = 0; c < 3; c++) {
      if (int rc = make_map(&m.own[c], g.F[(esweep ? EX : HX) + c], dt, e, w, jh)) return rc;
      if (int rc = make_map(&m.oth[c], g.F[(esweep ? HX : EX) + c], dt, e, wc, jh + 1)) return rc;
    }
    const int ncoef = esweep ? 6 : 3;
    const CoefIndex &ci = esweep ? cie : cih;
    if (ci.idx) {
      if (int rc = make_map(&m.idx, ci.idx, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, 32, jh)) return rc;
    } else {
      for (int c = 0; c < ncoef; c++)
        if (int rc = make_map(&m.coef[c], g.cf[(esweep ? 0 : 6) + c], dt, e, w, jh)) return rc;
    }
    if (has_pml) {
      const PmlFull<T> &pf = esweep ? pfe : pfh;
      for (int c = 0; c < (esweep ? 6 : 3); c++) {
        if (int rc = make_map(&m.aux[c], pf.aux[c], dt, e, w, jh)) return rc;
        if (m.wn > 0)
          if (int rc = make_map(&m.auxn[c], pf.aux[c], dt, e, m.wn, jh)) return rc;
      }
    }
    return 0;
  }




  // Per-tile headers (see SweepHeader): membership masks, line lengths and
  // UPML profiles, built on the device (k_headers) from the uploaded tiles
  // and the storage-type line and profile arrays the engine already holds.
  template <bool ES, bool PML>
  int build_headers(SweepLaunch &L)
  {
    using Hdr = SweepHeader<T, PML>;
    Hdr *d = nullptr;
    if (mem.alloc(&d, (size_t)L.ntiles)) return VGPU_ENOMEM;
    HeaderBoxes hb{};
    const Box *bb = ES ? be : bh;
    for (int c = 0; c < 3; c++) hb.bulk[c] = bb[c];
    for (int q = 0; q < pv.nreg; q++)
      for (int c = 0; c < 3; c++) hb.reg[q][c] = pv.lim[q][(ES ? EX : HX) + c];
    HeaderLines<T> hl{};
    for (int a = 0; a < 3; a++) {
      hl.line[a] = ES ? g.idh[a] : g.ide[a];
      hl.prof[0][a] = ES ? pv.ad[a] : pv.ah[a];
      hl.prof[1][a] = ES ? pv.bd[a] : pv.bh[a];
      hl.prof[2][a] = ES ? pv.ah[a] : pv.ad[a];
      hl.prof[3][a] = ES ? pv.ibh[a] : pv.ibd[a];
      hl.n[a] = p.n[a];
    }
    k_headers<T, ES, PML><<<L.ntiles, 32, 0, ss>>>(L.tiles, L.ntiles, hb, hl, d);
    CK(cudaGetLastError());
    L.headers = d;
    return 0;
  }

  template <bool ES, bool PML>
  int prepare_launch(SweepLaunch &L, const std::vector<SweepTile> &tiles, bool compressed)
  {
    L.ntiles = (int)tiles.size();
    if (!L.ntiles) return 0;
    for (const SweepTile &t : tiles)
      if (t.i1 - t.i0 + 1 > kSweepMaxPlanes || t.k0 % kSweepKW)
        return set_err(VGPU_EINVAL, "sweep tile of %d planes at k0=%d", t.i1 - t.i0 + 1, t.k0);
    if (upload(&L.tiles, tiles.data(), tiles.size())) return VGPU_ENOMEM;
    L.host = tiles;
    if (int rc = build_headers<ES, PML>(L)) return rc;
    L.smem = SweepLayout<T, ES, PML>::smem_bytes(compressed);
    auto kern = k_sweep_tma<T, ES, PML>;
    // The attribute is per kernel, shared by every engine in the process:
    // set it to the larger (uncompressed) layout.
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)SweepLayout<T, ES, PML>::smem_bytes(false)));
    int per_sm = 0, nsm = 148;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSweepThreads, L.smem));
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    if (per_sm < 1) return set_err(VGPU_ECUDA, "sweep kernel does not fit on an SM (%u bytes of shared memory)", L.smem);
    if (g_tune_blocks > 0) per_sm = std::min(per_sm, g_tune_blocks);
    L.grid = std::min(L.ntiles, per_sm * nsm);
    // Points each launch updates, for throughput accounting.
    const Box *bb = ES ? be : bh;
    for (const SweepTile &t : tiles) {
      const Box tb = tile_box(t);
      for (int c = 0; c < 3; c++) {
        if (t.bulk) L.bulk_points += box_overlap(tb, bb[c]);
        for (int r = 0; r < 2; r++)
          if (t.reg[r] >= 0) L.pml_points += box_overlap(tb, pv.lim[t.reg[r]][(ES ? EX : HX) + c]);
      }
    }
    return 0;
  }

  // Regions of one component must be disjoint from each other and from the
  // bulk box, so that full-volume auxiliaries hold each point's own state.
  int check_disjoint()
  {
    for (int f = 0; f < 6; f++) {
      const Box &bulk = f < 3 ? be[f] : bh[f - 3];
      for (int a = 0; a < pv.nreg; a++) {
        const Box &x = pv.lim[a][f];
        if (x.empty()) continue;
        auto meet = [](const Box &u, const Box &v) {
          return !u.empty() && !v.empty() && u.i0 <= v.i1 && v.i0 <= u.i1 && u.j0 <= v.j1 && v.j0 <= u.j1 &&
                 u.k0 <= v.k1 && v.k0 <= u.k1;
        };
        if (meet(x, bulk)) return set_err(VGPU_EINVAL, "PML region %d overlaps the bulk limits of field %d", a, f);
        for (int b = a + 1; b < pv.nreg; b++)
          if (meet(x, pv.lim[b][f])) return set_err(VGPU_EINVAL, "PML regions %d and %d overlap for field %d", a, b, f);
      }
    }
    return 0;
  }

  int setup_sweeps()
  {
    if (mem.alloc(&d_err, 1) || mem.alloc(&d_energy, 2)) return VGPU_ENOMEM;
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), ss));
    CK(cudaMemsetAsync(d_energy, 0, 2 * sizeof(double), ss));
    if (has_pml) {
      if (int rc = check_disjoint()) return rc;
      T *aux = nullptr;
      if (mem.alloc(&aux, (size_t)vol * 9)) return VGPU_ENOMEM;
      CK(cudaMemsetAsync(aux, 0, sizeof(T) * vol * 9, ss));
      for (int c = 0; c < 6; c++) pfe.aux[c] = aux + (int64_t)c * vol;
      for (int c = 0; c < 3; c++) pfh.aux[c] = aux + (int64_t)(6 + c) * vol;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    const int halo = 16 / (int)sizeof(T);
    const RegionSet rs = regions_of(p);
    for (int es = 0; es < 2; es++) {
      SweepPlan pl = plan_sweep(es ? ube : ubh, rs, es != 0, halo, nsm, g_tune_depth);
      (es ? maps_e : maps_h).wn = pl.wn;
      SweepLaunch *L = es ? sw_e : sw_h;
      const bool comp = (es ? cie : cih).idx != nullptr;
      mark("tiles");
      if (es) {
        if (int rc = prepare_launch<true, false>(L[0], pl.bulk, comp)) return rc;
        if (int rc = prepare_launch<true, true>(L[1], pl.pml, comp)) return rc;
      } else {
        if (int rc = prepare_launch<false, false>(L[0], pl.bulk, comp)) return rc;
        if (int rc = prepare_launch<false, true>(L[1], pl.pml, comp)) return rc;
      }
      mark("headers");
    }
    if (int rc = make_sweep_maps(maps_e, true)) return rc;
    if (int rc = make_sweep_maps(maps_h, false)) return rc;
    return 0;
  }

  // Launch one sweep kernel of a half step: which = 0 the bulk tiles, 1 the
  // UPML and mixed tiles.  Counts launched kernels through `count`.
  int launch_sweeps(bool esweep, int which, uint64_t *count, cudaStream_t st = nullptr)
  {
    if (!st) st = s;
    const dim3 blk(kSweepThreads);
    SweepLaunch &L = (esweep ? sw_e : sw_h)[which];
    if (!L.ntiles) return 0;
    const CoefIndex &ci = esweep ? cie : cih;
    const PmlFull<T> &pf = esweep ? pfe : pfh;
    const SweepMaps &mp = esweep ? maps_e : maps_h;
    if (esweep && which == 0)
      k_sweep_tma<T, true, false><<<L.grid, blk, L.smem, st>>>(mp, g, L.tiles, (const SweepHeader<T, false> *)L.headers,
                                                            L.ntiles, pf, ci, d_err);
    else if (esweep)
      k_sweep_tma<T, true, true><<<L.grid, blk, L.smem, st>>>(mp, g, L.tiles, (const SweepHeader<T, true> *)L.headers,
                                                           L.ntiles, pf, ci, d_err);
    else if (which == 0)
      k_sweep_tma<T, false, false><<<L.grid, blk, L.smem, st>>>(mp, g, L.tiles, (const SweepHeader<T, false> *)L.headers,
                                                             L.ntiles, pf, ci, d_err);
    else
      k_sweep_tma<T, false, true><<<L.grid, blk, L.smem, st>>>(mp, g, L.tiles, (const SweepHeader<T, true> *)L.headers,
                                                            L.ntiles, pf, ci, d_err);
    if (count) ++*count;
    return 0;
  }

  int setup_coef_index()
  {
    if (int rc = build_index(0, 6, cie)) return rc;
    mark("index-e");
    int rc = build_index(6, 3, cih);
    mark("index-h");
    return rc;
  }

  void setup_ghost()
  {
    int maxp = 1;
    for (int f = 0; f < 6; f++) {
      gv.mode[f] = p.ghost[f];
      if (p.ghost[f] != VGPU_GHOST_NONE) ghost_e = ghost_h = true;
    }
    for (int a = 0; a < 3; a++) {
      gv.go_lo[a] = p.gobox[2 * a];
      gv.go_hi[a] = p.gobox[2 * a + 1];
    }
    for (int a = 0; a < 3; a++) {
      int b = (a + 1) % 3, c = (a + 2) % 3;
      int np = (gv.go_hi[b] - gv.go_lo[b] + 2) * (gv.go_hi[c] - gv.go_lo[c] + 2);
      maxp = std::max(maxp, np);
    }
    ghost_threads = maxp;
  }

  // The last step sampled: the output window's end, or the problem's last
  // step if the window runs past it (samples beyond it have no buffer row).
  uint64_t out_last() const { return p.num_steps ? std::min<uint64_t>(p.out_stop, p.num_steps - 1) : 0; }

  int setup_observers()
  {
    if (p.num_steps > 0 && p.out_start < p.num_steps)
      nout = (p.out_stop < p.num_steps - 1 ? p.out_stop : p.num_steps - 1) - p.out_start + 1;
    if (upload(&d_td_pts, p.td_points, (size_t)p.num_td * 3) || upload(&d_fd_pts, p.fd_points, (size_t)p.num_fd * 3))
      return VGPU_ENOMEM;
    if (mem.alloc(&d_td, (size_t)nout * p.num_td * 6)) return VGPU_ENOMEM;
    size_t npc = (size_t)p.num_fd * 6;
    if (mem.alloc(&d_stage, npc * kStageRows) || mem.alloc(&d_re, npc * p.num_freq) ||
        mem.alloc(&d_im, npc * p.num_freq) || mem.alloc(&d_tw, (size_t)kTwRows * p.num_freq))
      return VGPU_ENOMEM;
    CK(cudaMemsetAsync(d_re, 0, sizeof(double) * (npc * p.num_freq ? npc * p.num_freq : 1), ss));
    CK(cudaMemsetAsync(d_im, 0, sizeof(double) * (npc * p.num_freq ? npc * p.num_freq : 1), ss));
    if (upload(&d_omega, p.omega, p.num_freq)) return VGPU_ENOMEM;
    return setup_bin();
  }

  int setup_bin()
  {
    if (p.num_bin <= 0) return 0;
    if (!p.bin_points) return set_err(VGPU_EINVAL, "num_bin > 0 with no bin_points");
    for (int64_t q = 0; q < p.num_bin; q++)
      for (int a = 0; a < 3; a++) {
        int v = p.bin_points[3 * q + a];
        if (v < 0 || v >= p.n[a]) return set_err(VGPU_EINVAL, "binary observer node %lld outside the grid", (long long)q);
      }
    size_t row = (size_t)p.num_bin * 6;
    if (upload(&d_bin_pts, p.bin_points, (size_t)p.num_bin * 3) || mem.alloc(&d_bin, 2 * kChunk * row))
      return VGPU_ENOMEM;
    CK(cudaMallocHost(&h_bin, sizeof(float) * 2 * kChunk * row));
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    for (int q = 0; q < 2; q++) {
      CK(cudaEventCreateWithFlags(&ev_fill[q], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&ev_copy[q], cudaEventDisableTiming));
    }
    return 0;
  }

  // A sweep block whose pipeline wait ran out leaves a code in d_err.
  int check_device_error()
  {
    int h = 0;
    CK(cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) return set_err(VGPU_ETIMEOUT, "a sweep's shared-memory pipeline timed out waiting for its loads");
    return 0;
  }

  // Hand the rows of ring block q to the sink once their copy has landed.
  int bin_deliver(int q)
  {
    BinBlock &b = bin_blk[q];
    if (!b.pending) return 0;
    b.pending = false;
    CK(cudaEventSynchronize(ev_copy[q]));
    size_t row = (size_t)p.num_bin * 6;
    const float *rows = h_bin + ((size_t)q * kChunk + (b.row0 + p.out_start) % kChunk) * row;
    if (bin_sink) bin_sink(bin_user, b.row0, b.nrows, p.num_bin, rows);
    return 0;
  }

  // Copy output steps lo..hi (absolute, inside one aligned chunk) of ring
  // block q to pinned host memory on the copy stream.
  int bin_enqueue(int q, uint64_t lo, uint64_t hi)
  {
    size_t row = (size_t)p.num_bin * 6;
    size_t off = ((size_t)q * kChunk + lo % kChunk) * row;
    CK(cudaEventRecord(ev_fill[q], s));
    CK(cudaStreamWaitEvent(cs, ev_fill[q], 0));
    CK(cudaMemcpyAsync(h_bin + off, d_bin + off, sizeof(float) * (hi - lo + 1) * row, cudaMemcpyDeviceToHost, cs));
    CK(cudaEventRecord(ev_copy[q], cs));
    bin_blk[q] = BinBlock{ true, lo - p.out_start, (uint32_t)(hi - lo + 1) };
    return 0;
  }

  static unsigned blocks_for(int64_t n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

  // The sweep of a half step: one launch, the UPML kernel over every tile
  // when the mesh has UPML regions, else the bulk kernel.
  int launch_sweep_pair(bool esweep, uint64_t *count)
  {
    if (int rc = launch_sweeps(esweep, 1, count)) return rc;
    return launch_sweeps(esweep, 0, count);
  }

  // Threads of one k_tfsf_list launch.
  static int64_t tfsf_threads(const TfsfList<T> &l)
  {
    return (l.nsingle + kTfsfPerThread - 1) / kTfsfPerThread + l.nmulti;
  }

  // The parts of one time step, in the order of src/simulation.c:156-222.
  // launch_part queues one part `rel` steps past the device step counter
  // (nothing when the problem has no such work) and counts its kernels.
  enum Part {
    P_OBSERVE, P_BIN, P_MUR_E, P_SWEEP_E, P_DEBYE, P_SIBC_E, P_SRC_E, P_TFSF_E, P_GHOST_E,
    P_MUR_H, P_SWEEP_H, P_SIBC_H, P_SRC_H, P_TFSF_H, P_GHOST_H, P_COUNT
  };

  bool part_present(int part) const
  {
    switch (part) {
      case P_OBSERVE: return p.num_td || p.num_fd;
      case P_BIN: return p.num_bin > 0;
      case P_MUR_E: return mve.nitems > 0;
      case P_SWEEP_E: return sw_e[0].ntiles || sw_e[1].ntiles;
      case P_DEBYE: return n_debye > 0;
      case P_SIBC_E: return nsibc > 0;
      case P_SRC_E:
      case P_SRC_H:
        for (const auto &l : srcs)
          if ((l.c <= EZ) == (part == P_SRC_E)) return true;
        return false;
      case P_TFSF_E:
      case P_TFSF_H:
        for (const auto &w : pws)
          if (w.pv.use_aux || (part == P_TFSF_E ? w.total_e : w.total_h)) return true;
        return false;
      case P_GHOST_E: return ghost_e;
      case P_MUR_H: return mvh.nitems > 0;
      case P_SWEEP_H: return sw_h[0].ntiles || sw_h[1].ntiles;
      case P_SIBC_H: return nsibc > 0 && ntgt > 0;
      case P_GHOST_H: return ghost_h;
      default: return false;
    }
  }

  int launch_part(int part, int rel, uint64_t *count)
  {
    uint64_t launches = 0;
    switch (part) {
      case P_OBSERVE:
        if (p.num_td || p.num_fd) {
          int nt = (p.num_td + p.num_fd) * 6;
          k_observe<T><<<blocks_for(nt, 128), 128, 0, s>>>(g, d_td_pts, p.num_td, d_fd_pts, p.num_fd, d_td, d_stage,
                                                            d_step, rel, p.out_start, out_last(), kStageRows);
          launches++;
        }
        break;
      case P_BIN:
        if (p.num_bin > 0) {
          k_bin_observe<T><<<blocks_for(p.num_bin * 6, 128), 128, 0, s>>>(g, d_bin_pts, p.num_bin, d_bin, d_step,
                                                                          rel, p.out_start, out_last(), kChunk);
          launches++;
        }
        break;
      // Mur reads the neighbours' pre-update E, so it precedes the sweeps;
      // the PML and bulk sweeps touch disjoint E points.
      case P_MUR_E:
        if (mve.nitems) {
          k_mur_e<T><<<dim3(blocks_for(mur_max_e, 128), mve.nitems), 128, 0, s>>>(g, mve);
          launches++;
        }
        break;
      case P_SWEEP_E:
        if (int rc = launch_sweep_pair(true, &launches)) return rc;
        break;
      case P_DEBYE:
        if (n_debye) {
          k_debye<T><<<blocks_for(debye_total, 128), 128, 0, s>>>(g, d_debye, n_debye, debye_total, d_J, d_lastE,
                                                                  d_dcoef);
          launches++;
        }
        break;
      case P_SIBC_E:
        if (nsibc) {
          k_sibc_e<T><<<blocks_for(sibc_faces, 128), 128, 0, s>>>(g, d_surfs, nsibc, d_models, d_q0, d_q1, d_q2,
                                                                  d_adjA, d_adjB, d_zofs, d_zeta, d_old, d_etan,
                                                                  sibc_faces);
          launches++;
        }
        break;
      case P_SRC_E:
      case P_SRC_H:
        for (auto &l : srcs)
          if ((l.c <= EZ) == (part == P_SRC_E)) {
            k_source<T><<<blocks_for(l.b.count(), 128), 128, 0, s>>>(g, l.b, l.c, l.kind, (T)l.soft,
                                                                     (const T *)l.values, d_step, rel);
            launches++;
          }
        break;
      case P_TFSF_E:
        for (auto &w : pws) {
          if (w.pv.use_aux) { k_aux_e<T><<<1, 256, 0, s>>>(w.pv, d_step, rel); launches++; }
          if (w.total_e) {
            k_tfsf_list<T><<<blocks_for(tfsf_threads(w.le), 128), 128, 0, s>>>(g, w.pv, w.te, w.le, p.dt, d_step,
                                                                                rel, 1);
            launches++;
          }
        }
        break;
      case P_GHOST_E:
        if (ghost_e) {
          k_ghost<T><<<dim3(blocks_for(ghost_threads, 128), 6), 128, 0, s>>>(g, gv, 1, 0);
          launches++;
        }
        break;
      case P_MUR_H:
        if (mvh.nitems) {
          k_mur_h<T><<<dim3(blocks_for(mur_max_h, 128), mvh.nitems), 128, 0, s>>>(g, mvh);
          launches++;
        }
        break;
      case P_SWEEP_H:
        if (int rc = launch_sweep_pair(false, &launches)) return rc;
        break;
      case P_SIBC_H:
        if (nsibc && ntgt) {
          k_sibc_h<T><<<blocks_for(ntgt, 128), 128, 0, s>>>(g, d_tgt_index, d_tgt_comp, d_tgt_start, ntgt, d_ops,
                                                            d_etan);
          launches++;
        }
        break;
      case P_TFSF_H:
        for (auto &w : pws) {
          if (w.pv.use_aux) { k_aux_h<T><<<1, 256, 0, s>>>(w.pv); launches++; }
          if (w.total_h) {
            k_tfsf_list<T><<<blocks_for(tfsf_threads(w.lh), 128), 128, 0, s>>>(g, w.pv, w.th, w.lh, p.dt, d_step,
                                                                                rel, 0);
            launches++;
          }
        }
        break;
      case P_GHOST_H:
        if (ghost_h) {
          k_ghost<T><<<dim3(blocks_for(ghost_threads, 128), 12), 128, 0, s>>>(g, gv, 0, 0);
          launches++;
        }
        break;
      default: return set_err(VGPU_EINVAL, "no step part %d", part);
    }
    if (count) *count += launches;
    return 0;
  }

  // Side launches that may share one kernel: the Debye update and the plane
  // wave's E corrections follow the E sweep with nothing between them when
  // there are no SIBC surfaces or E sources, and the plane wave's H
  // corrections end the step when there is no ghost layer.  They share a
  // launch only if they touch disjoint points -- no Debye cell of a component
  // is a corrected point of it; no observer point is a corrected H point --
  // so that their order does not matter.  Observer samples taken with the H
  // corrections are those of the next step (src/observer.c:622-650 samples
  // at the top of a step, i.e. the fields as the previous step left them).
  void plan_side_merges()
  {
    bool e_src = false;
    for (const auto &l : srcs) e_src = e_src || l.c <= EZ;
    if (pws.size() == 1 && n_debye && pws[0].total_e && !nsibc && !e_src) {
      bool disjoint = true;
      for (int b = 0; b < p.num_debye && disjoint; b++)
        for (int c = 0; c < 3 && disjoint; c++)
          for (int q = 0; q < pws[0].te.n && disjoint; q++)
            if (pws[0].te.it[q].c == c && boxes_meet(box_from(p.debye[b].flim[c]), pws[0].te.it[q].b)) disjoint = false;
      merge_e = disjoint;
    }
    if (pws.size() == 1 && (p.num_td || p.num_fd) && p.num_bin <= 0 && pws[0].total_h && !ghost_h) {
      bool disjoint = true;
      for (int q = 0; q < pws[0].th.n && disjoint; q++) {
        const Box &b = pws[0].th.it[q].b;
        for (int t = 0; t < p.num_td && disjoint; t++)
          if (b.contains(p.td_points[3 * t], p.td_points[3 * t + 1], p.td_points[3 * t + 2])) disjoint = false;
        for (int t = 0; t < p.num_fd && disjoint; t++)
          if (b.contains(p.fd_points[3 * t], p.fd_points[3 * t + 1], p.fd_points[3 * t + 2])) disjoint = false;
      }
      merge_obs = disjoint;
    }
    if (merge_e) {
      SideLaunch<T> &L = side_e;
      L.nb_debye = (int)blocks_for(debye_total, 128);
      L.nb_tfsf = (int)blocks_for(tfsf_threads(pws[0].le), 128);
      L.debye = d_debye; L.n_debye = n_debye; L.debye_total = debye_total;
      L.J = d_J; L.lastE = d_lastE; L.dcoef = d_dcoef;
      L.pw = pws[0].pv; L.tv = pws[0].te; L.tl = pws[0].le; L.dt = p.dt; L.efield = 1;
    }
    if (merge_obs) {
      SideLaunch<T> &L = side_h;
      L.nb_tfsf = (int)blocks_for(tfsf_threads(pws[0].lh), 128);
      L.nb_obs = (int)blocks_for((int64_t)(p.num_td + p.num_fd) * 6, 128);
      L.pw = pws[0].pv; L.tv = pws[0].th; L.tl = pws[0].lh; L.dt = p.dt; L.efield = 0;
      L.td_pts = d_td_pts; L.num_td = p.num_td; L.fd_pts = d_fd_pts; L.num_fd = p.num_fd;
      L.td_buf = d_td; L.fd_stage = d_stage; L.out_start = p.out_start; L.out_stop = out_last();
      L.tblock = kStageRows;
    }
    stats.merged_parts = (merge_e ? 1u : 0u) | (merge_obs ? 2u : 0u);
  }

  // Whether the step launches anything for a part, merges included.
  bool step_part_present(int part) const
  {
    if (merge_obs && part == P_OBSERVE) return false;
    if (merge_e && part == P_TFSF_E) return pws[0].pv.use_aux != 0;
    return part_present(part);
  }

  // One part as the step launches it: with merge_e the Debye part is the
  // merged launch (after the auxiliary grid's E update, which the
  // corrections read) and the TFSF E part is empty; with merge_obs the
  // observer part is empty (the previous step's last launch took the
  // samples) and the TFSF H part is the merged launch.
  int launch_step_part(int part, int rel, uint64_t *count)
  {
    uint64_t launches = 0;
    if (merge_e && (part == P_DEBYE || part == P_TFSF_E)) {
      if (part == P_DEBYE) {
        if (pws[0].pv.use_aux) { k_aux_e<T><<<1, 256, 0, s>>>(pws[0].pv, d_step, rel); launches++; }
        k_side<T><<<side_e.nb_debye + side_e.nb_tfsf, 128, 0, s>>>(g, side_e, d_step, rel);
        launches++;
      }
    } else if (merge_obs && (part == P_OBSERVE || part == P_TFSF_H)) {
      if (part == P_TFSF_H) {
        if (pws[0].pv.use_aux) { k_aux_h<T><<<1, 256, 0, s>>>(pws[0].pv); launches++; }
        k_side<T><<<side_h.nb_tfsf + side_h.nb_obs, 128, 0, s>>>(g, side_h, d_step, rel);
        launches++;
      }
    } else {
      return launch_part(part, rel, count);
    }
    if (count) *count += launches;
    return 0;
  }

  int enqueue_step(int rel)
  {
    uint64_t launches = 0;
    for (int part = 0; part < P_COUNT; part++)
      if (int rc = launch_step_part(part, rel, &launches)) return rc;
    launches_per_step = launches;
    return 0;
  }

  // `m` steps and the counter's advance past them.
  int enqueue_steps(int m)
  {
    for (int q = 0; q < m; q++)
      if (int rc = enqueue_step(q)) return rc;
    k_advance<<<1, 1, 0, s>>>(d_step, m);
    return 0;
  }

  // Graph q holds kGraphSteps >> q steps (16, 8, 4, 2, 1) and the counter's
  // advance past them.  The 16-step graph is captured at creation, the
  // shorter ones on first use: a block that does not start on a 16-step
  // boundary (a run of any length, a service's partial block) is replayed
  // from graphs too, largest first, instead of single kernel launches.
  static constexpr int kNumGraphs = 5;

  int capture_graph(int q = 0)
  {
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_steps(kGraphSteps >> q);
    const cudaError_t ee = cudaStreamEndCapture(s, &gr);
    if (rc) {
      if (ee == cudaSuccess && gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (ee != cudaSuccess) return set_err(VGPU_ECUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ee));
    const cudaError_t e = cudaGraphInstantiate(&graphs[q], gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
      graphs[q] = nullptr;
      return set_err(VGPU_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    }
    return 0;
  }

  // m steps as graph launches, largest graphs first.
  int launch_graphs(uint64_t m)
  {
    for (int q = 0; q < kNumGraphs && m; q++) {
      const uint64_t len = (uint64_t)(kGraphSteps >> q);
      while (m >= len) {
        if (!graphs[q])
          if (int rc = capture_graph(q)) return rc;
        CK(cudaGraphLaunch(graphs[q], s));
        stats.kernel_launches += len * launches_per_step + 1;
        m -= len;
      }
    }
    return 0;
  }

  // Accumulate the DFT of output rows [r0, r1) (one chunk at most).
  int dft_rows(uint64_t r0, uint64_t r1)
  {
    if (!p.num_fd || r1 <= r0) return 0;
    int nrows = (int)(r1 - r0);
    int nf = p.num_freq, npc = p.num_fd * 6;
    k_twiddle<<<blocks_for((int64_t)nrows * nf, 128), 128, 0, s>>>(d_omega, nf, p.dt, p.out_start, r0, nrows, d_tw);
    const int tiles = (npc + kDftTileM - 1) / kDftTileM;
    for (int t0 = 0; t0 < tiles; t0 += 65535) {
      const dim3 grd((nf + kDftTileF - 1) / kDftTileF, std::min(65535, tiles - t0));
      k_dft_mma<<<grd, 128, 0, s>>>(d_stage, npc, nf, nrows, (int)(r0 % kStageRows), kStageRows, d_tw, d_re, d_im,
                                    t0 * kDftTileM);
      stats.kernel_launches += 1;
    }
    stats.kernel_launches += 1;
    return 0;
  }

  // Queue the next block of at most max_steps steps (up to the next 64-step
  // boundary, replayed from the step graphs) on the engine's stream, with the block's DFT fold and binary-row copy; *queued
  // gets the count.
  int issue_block(uint64_t max_steps, uint64_t *queued)
  {
    const uint64_t n0 = step;
    // Blocks stay aligned so the DFT staging rows of one block never wrap.
    const uint64_t room = kChunk - (n0 % kChunk);
    const uint64_t m = std::min<uint64_t>(room, max_steps);
    *queued = 0;
    if (!m) return 0;
    const int q = (int)((n0 / kChunk) & 1);
    // The ring block this chunk fills last held the chunk two back: hand
    // those rows over (the device is busy with the previous chunk) before
    // they are overwritten.
    if (p.num_bin > 0)
      if (int rc = bin_deliver(q)) return rc;
    // With merged observer sampling each step samples the next one; the
    // first step of a problem, and a step whose fields were overwritten
    // after its samples were taken, are sampled here.
    if (merge_obs && need_sample) {
      if (int rc = launch_part(P_OBSERVE, 0, &stats.kernel_launches)) return rc;
      need_sample = false;
    }
    if (int rc = launch_graphs(m)) return rc;
    if (int rc = after_block(n0, m, q)) return rc;
    *queued = m;
    return 0;
  }

  // The work that follows a block of m steps from step n0 (the block's
  // steps are queued on s): binary rows, the DFT fold and the energy check.
  int after_block(uint64_t n0, uint64_t m, int q)
  {
    step = n0 + m;
    // Output rows produced in this block.
    const uint64_t lo = std::max<uint64_t>(n0, p.out_start), hi = std::min<uint64_t>(step - 1, p.out_stop);
    if (p.num_bin > 0 && bin_sink && hi >= lo && lo <= p.out_stop) {
      if (int rc = bin_enqueue(q, lo, hi)) return rc;
    }
    // The staged rows are folded into the running DFT once their 64-step
    // chunk is complete (or the problem ends); rows of a chunk that a run
    // leaves unfinished are folded with the rest of the chunk, or when the
    // DFT is read.  A fold costs about the same for 20 rows as for 64 (it
    // reads and writes every running sum), so partial chunks are not folded
    // early.
    if (p.num_fd && (step % kChunk == 0 || step == p.num_steps))
      if (int rc = fold_pending()) return rc;
    if (step % kChunk == 0 || step == p.num_steps)
      if (int rc = queue_energy()) return rc;
    return 0;
  }

  // Whether the engine can step in a group (k_sweep_tma<..., GROUP>,
  // k_group_side): its steps hold only sweeps, point sources and point
  // observers, its coefficients are indexed with at most kGroupTab tuples,
  // and each half step's tiles belong to one sweep kernel.
  bool groupable() const
  {
    if (!cie.idx || !cih.idx || cie.ntab > kGroupTab || cih.ntab > kGroupTab) return false;
    if (mve.nitems || mvh.nitems || n_debye || nsibc || !pws.empty() || ghost_e || ghost_h || p.num_bin > 0)
      return false;
    if (merge_e || merge_obs) return false;
    for (const SweepLaunch *L : { sw_e, sw_h })
      if (L[0].ntiles && L[1].ntiles) return false;
    return true;
  }

  // The sweep kernel class of a half step's tiles: 0 the bulk kernel, 1
  // the UPML kernel, -1 none.
  int sweep_class(bool es) const
  {
    const SweepLaunch *L = es ? sw_e : sw_h;
    return L[1].ntiles ? 1 : L[0].ntiles ? 0 : -1;
  }

  // Fold every staged output row of the steps run so far that is not yet in
  // the running DFT (at most one chunk: folds happen at every chunk end).
  int fold_pending()
  {
    if (!p.num_fd || step <= p.out_start) return 0;
    const uint64_t staged = std::min<uint64_t>(step - 1, out_last()) - p.out_start + 1;
    if (staged <= dft_folded) return 0;
    if (int rc = dft_rows(dft_folded, staged)) return rc;
    dft_folded = staged;
    return 0;
  }

  // The stability check of the fields as they stand after the queued steps.
  int queue_energy()
  {
    CK(cudaMemsetAsync(d_energy, 0, 2 * sizeof(double), s));
    k_energy<T><<<4 * 148, 256, 0, s>>>(g, vol, d_energy);
    stats.kernel_launches += 1;
    energy_step = step;
    return 0;
  }

  // After the queued work has finished: errors, then the binary rows still
  // pending, older block first.
  int finish_queued()
  {
    if (int rc = check_device_error()) return rc;
    if (energy_step) {
      double en[2] = { 0, 0 };
      CK(cudaMemcpy(en, d_energy, sizeof en, cudaMemcpyDeviceToHost));
      stats.energy_e = en[0];
      stats.energy_h = en[1];
      stats.energy_step = energy_step;
      if (!std::isfinite(en[0]) || !std::isfinite(en[1]))
        return set_err(VGPU_ENONFINITE, "the fields' FP64 sums of squares are not finite at step %llu",
                       (unsigned long long)energy_step);
    }
    if (p.num_bin > 0) {
      int a = 0, b = 1;
      if (bin_blk[1].pending && (!bin_blk[0].pending || bin_blk[1].row0 < bin_blk[0].row0)) a = 1, b = 0;
      if (int rc = bin_deliver(a)) return rc;
      if (int rc = bin_deliver(b)) return rc;
    }
    CK(cudaGetLastError());
    return 0;
  }

  int check_steps(uint64_t nsteps) override
  {
    if (step + nsteps > p.num_steps)
      return set_err(VGPU_EINVAL, "run of %llu steps from step %llu exceeds the problem's %llu steps",
                     (unsigned long long)nsteps, (unsigned long long)step, (unsigned long long)p.num_steps);
    return 0;
  }

  int run(uint64_t nsteps) override
  {
    if (int rc = check_steps(nsteps)) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
    stats.kernel_launches = 0;
    for (uint64_t done = 0; done < nsteps;) {
      uint64_t m = 0;
      if (int rc = issue_block(nsteps - done, &m)) return rc;
      done += m;
    }
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    if (int rc = finish_queued()) return rc;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    stats.run_ms = ms;
    stats.steps = nsteps;
    return 0;
  }

  // Up to max_steps more steps, never past the problem's last step.
  int enqueue(uint64_t max_steps, uint64_t *queued) override
  {
    const uint64_t left = step < p.num_steps ? p.num_steps - step : 0;
    return issue_block(std::min<uint64_t>(max_steps, left), queued);
  }

  // 1: the queued work has finished; 0: still running; a device error
  // (sticky or not) is reported, never read as "still running".
  int query() override
  {
    const cudaError_t e = cudaStreamQuery(s);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return set_err(VGPU_ECUDA, "stream query: %s", cudaGetErrorString(e));
  }

  int synchronize() override
  {
    CK(cudaStreamSynchronize(s));
    return finish_queued();
  }

  int read_td(double *out, uint64_t steps) override
  {
    size_t n = (size_t)std::min<uint64_t>(steps, nout) * p.num_td * 6;
    std::vector<T> tmp(n ? n : 1);
    if (n) {
      CK(cudaStreamSynchronize(s));
      if (int rc = pinned_stage().d2h(tmp.data(), d_td, sizeof(T) * n, s)) return rc;
    }
    for (size_t q = 0; q < n; q++) out[q] = (double)tmp[q];
    return 0;
  }

  int read_dft(double *re, double *im) override
  {
    size_t n = (size_t)p.num_fd * 6 * p.num_freq;
    if (!n) return 0;
    if (int rc = fold_pending()) return rc;
    CK(cudaStreamSynchronize(s));
    // Into page-locked memory the sums go straight from the device.
    if (is_pinned(re) && is_pinned(im)) {
      CK(cudaMemcpyAsync(re, d_re, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(im, d_im, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    } else {
      if (int rc = pinned_stage().d2h(re, d_re, sizeof(double) * n, s)) return rc;
      if (int rc = pinned_stage().d2h(im, d_im, sizeof(double) * n, s)) return rc;
    }
    return 0;
  }

  int read_field(int c, double *out) override
  {
    std::vector<T> tmp((size_t)vol);
    CK(cudaStreamSynchronize(s));
    if (int rc = pinned_stage().d2h(tmp.data(), g.F[c], sizeof(T) * vol, s)) return rc;
    for (int i = 0; i < p.n[0]; i++)
      for (int j = 0; j < p.n[1]; j++)
        for (int k = 0; k < p.n[2]; k++)
          out[((int64_t)i * p.n[1] + j) * p.n[2] + k] = (double)tmp[(int64_t)i * g.s0 + (int64_t)j * g.s1 + k];
    return 0;
  }

  int write_field(int c, const double *in) override
  {
    CK(cudaStreamSynchronize(s));
    need_sample = true;
    if (int rc = upload_volume(g.F[c], in)) return rc;
    CK(cudaStreamSynchronize(ss));
    return 0;
  }

  // Launch one sweep over its tile list; with `required` an empty list is an
  // error (profiling), otherwise it launches nothing.
  int launch_one(int kernel, bool required = true, uint64_t *count = nullptr)
  {
    const bool es = kernel == VGPU_K_BULK_E || kernel == VGPU_K_PML_E;
    const int which = (kernel == VGPU_K_BULK_E || kernel == VGPU_K_BULK_H) ? 0 : 1;
    const SweepLaunch *L = es ? sw_e : sw_h;
    const bool present = L[which].ntiles > 0;
    if (kernel < 0 || kernel > 3 || !present) {
      if (!required) return 0;
      return set_err(VGPU_EINVAL, "kernel %d not present in this problem", kernel);
    }
    return launch_sweeps(es, which, count);
  }

  int sweep_points(int kernel, uint64_t *bulk_pts, uint64_t *pml_pts) override
  {
    if (kernel < 0 || kernel > 3) return set_err(VGPU_EINVAL, "kernel %d is not a sweep", kernel);
    const bool es = kernel == VGPU_K_BULK_E || kernel == VGPU_K_PML_E;
    const SweepLaunch &L = (es ? sw_e : sw_h)[(kernel == VGPU_K_BULK_E || kernel == VGPU_K_BULK_H) ? 0 : 1];
    *bulk_pts = L.bulk_points;
    *pml_pts = L.pml_points;
    return 0;
  }

  // The step part a VGPU_K_* id above the sweeps names (-1: none).
  static int part_of(int kernel)
  {
    static const int map[] = { P_OBSERVE, P_BIN, P_MUR_E, P_DEBYE, P_SIBC_E, P_SRC_E, P_TFSF_E, P_GHOST_E,
                               P_MUR_H, P_SIBC_H, P_SRC_H, P_TFSF_H, P_GHOST_H };
    const int q = kernel - VGPU_K_OBSERVE;
    return q >= 0 && q < (int)(sizeof map / sizeof map[0]) ? map[q] : -1;
  }

  // One launch of a timed kernel: a sweep, a step part or a 64-row DFT fold.
  int launch_timed(int kernel)
  {
    if (kernel >= 0 && kernel <= 3) return launch_one(kernel);
    if (kernel == VGPU_K_DFT_BLOCK) {
      const uint64_t st = stats.kernel_launches;
      const int rc = dft_rows(0, kTwRows);
      stats.kernel_launches = st;
      return rc;
    }
    if (kernel == VGPU_K_DFT_BLOCK_SCALAR) {
      const int nf = p.num_freq, npc = p.num_fd * 6;
      k_twiddle<<<blocks_for((int64_t)kTwRows * nf, 128), 128, 0, s>>>(d_omega, nf, p.dt, p.out_start, 0, kTwRows,
                                                                       d_tw);
      const dim3 blk(32, 8), grd((nf + 31) / 32, (npc + 7) / 8);
      if (grd.y > 65535) return set_err(VGPU_EINVAL, "%d point-components exceed the scalar fold's grid", npc);
      k_dft_accumulate<<<grd, blk, sizeof(double) * 8 * kTwRows, s>>>(d_stage, npc, nf, kTwRows, 0, kStageRows, d_tw,
                                                                     d_re, d_im);
      return 0;
    }
    return launch_step_part(part_of(kernel), 0, nullptr);
  }

  int time_kernel(int kernel, int warmup, int iters, double *ms, uint64_t *points) override
  {
    // Timed launches act at the current step (the counter does not move);
    // step-indexed tables (source values, the auxiliary grid's drive) have
    // rows for the problem's steps only.
    if (step >= p.num_steps) return set_err(VGPU_EINVAL, "kernel timing needs a step inside the problem");
    uint64_t pts = 0;
    if (kernel >= 0 && kernel <= 3) {
      uint64_t bulk_pts = 0, pml_pts = 0;
      if (int rc = sweep_points(kernel, &bulk_pts, &pml_pts)) return rc;
      pts = bulk_pts + pml_pts;
      const bool es = kernel == VGPU_K_BULK_E || kernel == VGPU_K_PML_E;
      if (!(es ? sw_e : sw_h)[(kernel == VGPU_K_BULK_E || kernel == VGPU_K_BULK_H) ? 0 : 1].ntiles)
        return set_err(VGPU_EINVAL, "kernel %d not present in this problem", kernel);
    } else if (kernel == VGPU_K_DFT_BLOCK || kernel == VGPU_K_DFT_BLOCK_SCALAR) {
      if (!p.num_fd) return set_err(VGPU_EINVAL, "kernel %d not present in this problem", kernel);
    } else {
      const int part = part_of(kernel);
      if (part < 0) return set_err(VGPU_EINVAL, "kernel %d is not a step kernel", kernel);
      if (!step_part_present(part)) return set_err(VGPU_EINVAL, "kernel %d not present in this problem", kernel);
    }
    for (int q = 0; q < warmup; q++)
      if (int rc = launch_timed(kernel)) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
    for (int q = 0; q < iters; q++)
      if (int rc = launch_timed(kernel)) return rc;
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    CK(cudaGetLastError());
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = iters > 0 ? t / iters : 0.0;
    *points = pts;
    return 0;
  }

  int check_finite() override
  {
    int *flag;
    if (mem.alloc(&flag, 1)) return VGPU_ENOMEM;
    CK(cudaMemsetAsync(flag, 0, sizeof(int), s));
    k_finite<T><<<592, 256, 0, s>>>(g, vol, flag);
    int h = 0;
    CK(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return h ? set_err(VGPU_ENONFINITE, "non-finite field value found") : 0;
  }
};

// ---- grouped stepping ----------------------------------------------------
//
// Many engines of one precision stepped together (the batched form of
// src/simulation.c:136-231's loop): per half step one launch of the grouped
// sweep kernel per sweep class over every member's tiles, and one
// k_group_side launch each for the members' samples, E sources and H
// sources -- a step of the whole group is at most seven launches however
// many meshes it holds -- replayed from captured graphs of 16, 8, 4, 2 and 1
// steps.  Members are ordered by steps left, most first, and every list
// (tiles, side items, step counters) follows that order; members finish from
// the end of the order, so the group of the first R members is a prefix of
// each list and a finished member leaves by shortening the launches (new
// graphs), with nothing copied.  The sweep blocks take chunks of tiles from
// a counter per launch (zeroed at each graph's start), so a launch ends
// evenly.  Every member's kernels do what its own step graph does, in the
// same order, on its own arrays, so its results are those of vgpu_run
// alone.

struct GroupBase {
  virtual ~GroupBase() {}
  virtual bool busy() const = 0;
  virtual int issue_block() = 0;
  virtual int finish() = 0;
  uint64_t launches = 0;
  int rebuilds = 0, members_at_start = 0;
  int64_t tiles_at_start = 0;
  double ms = 0;
};

template <typename T>
struct Group : GroupBase {
  struct Member {
    Engine<T> *e;
    uint64_t left;
  };
  // The launches of the first R members, as graphs.
  struct View {
    int R = 0;
    int grid[2][2] = {}, ntiles[2][2] = {};
    cudaGraphExec_t graphs[5] = {};
    uint64_t per_step = 0;        // launches of one step
    cudaEvent_t done = nullptr;   // after this view's last launch
  };
  std::vector<Member> members;   // by steps left, most first; the first R are active
  int R = 0;
  DevAlloc da;
  // Device lists, in member order, and the prefix counts per member count.
  GroupMesh<T> *meshes[2][2] = {};   // [E, H][sweep class]
  GroupTile *tiles[2][2] = {};
  std::vector<int> tiles_upto[2][2];   // tiles of the first r members, r = 0..n
  int *counters = nullptr;             // one per sweep launch of a graph
  int chunk = 4;                       // tiles a sweep block takes at a time
  GroupSide<T> *side[3] = {};        // samples, E sources, H sources
  std::vector<int> side_upto[3], blk_upto[3];
  uint64_t **steps = nullptr;
  char *host = nullptr;   // pinned image of the lists
  View *cur = nullptr;
  std::vector<View *> retired;
  cudaStream_t s = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  int *d_err = nullptr;
  int nsm = 148;
  int per_sm[2][2] = {};
  std::vector<Engine<T> *> all;   // every member the group started with

  ~Group() override
  {
    if (s) cudaStreamSynchronize(s);
    if (cur) release(cur);
    for (View *v : retired) release(v);
    if (host) cudaFreeHost(host);
    da.free_all();
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (s) cudaStreamDestroy(s);
  }

  bool busy() const override { return R > 0; }

  template <bool ES, bool PML>
  int kernel_setup(int h, int c)
  {
    auto kern = k_sweep_tma<T, ES, PML, true>;
    const uint32_t smem = SweepLayout<T, ES, PML>::smem_bytes(true);
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int n = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, kSweepThreads, smem));
    if (n < 1) return set_err(VGPU_ECUDA, "grouped sweep kernel does not fit on an SM (%u bytes of shared memory)", smem);
    if (g_tune_blocks > 0) n = std::min(n, g_tune_blocks);
    per_sm[h][c] = n;
    return 0;
  }

  void release(View *v)
  {
    for (auto &g : v->graphs)
      if (g) cudaGraphExecDestroy(g);
    if (v->done) cudaEventDestroy(v->done);
    delete v;
  }

  // Streams, flags and the lists; the members' earlier work is finished
  // first (collect synchronised them).
  int start()
  {
    std::stable_sort(members.begin(), members.end(), [](const Member &a, const Member &b) { return a.left > b.left; });
    const int n = (int)members.size();
    R = members_at_start = n;
    for (Member &mb : members) {
      all.push_back(mb.e);
      mb.e->stats.steps = 0;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    if (int rc = kernel_setup<true, false>(0, 0)) return rc;
    if (int rc = kernel_setup<true, true>(0, 1)) return rc;
    if (int rc = kernel_setup<false, false>(1, 0)) return rc;
    if (int rc = kernel_setup<false, true>(1, 1)) return rc;
    // Layout of one device buffer: each list 256-byte aligned.
    size_t off = 0;
    auto place = [&](size_t bytes) {
      const size_t o = off;
      off = (off + bytes + 255) / 256 * 256;
      return o;
    };
    const size_t o_err = place(sizeof(int));
    const size_t o_counters = place(sizeof(int) * kGraphSteps * 4);
    if (g_tune_chunk > 0) chunk = g_tune_chunk;
    size_t o_mesh[2][2], o_tiles[2][2];
    std::vector<int> cls_index[2][2];   // member q's index in its class's mesh array
    for (int h = 0; h < 2; h++)
      for (int c = 0; c < 2; c++) {
        int nm = 0, nt = 0;
        tiles_upto[h][c].assign(1, 0);
        cls_index[h][c].assign(n, -1);
        for (int q = 0; q < n; q++) {
          Engine<T> *e = members[q].e;
          if (e->sweep_class(h == 0) == c) {
            cls_index[h][c][q] = nm++;
            nt += (h == 0 ? e->sw_e : e->sw_h)[c].ntiles;
          }
          tiles_upto[h][c].push_back(nt);
        }
        o_mesh[h][c] = place(sizeof(GroupMesh<T>) * (size_t)nm);
        o_tiles[h][c] = place(sizeof(GroupTile) * (size_t)nt);
        tiles_at_start += nt;
      }
    std::vector<size_t> o_tab(2 * (size_t)n);
    for (int q = 0; q < n; q++)
      for (int h = 0; h < 2; h++) {
        const CoefIndex &ci = h == 0 ? members[q].e->cie : members[q].e->cih;
        o_tab[2 * q + h] = place((size_t)ci.ntab * (h == 0 ? 6 : 3) * sizeof(T));
      }
    std::vector<GroupSide<T>> items[3];
    std::vector<int> owner[3];
    for (int k = 0; k < 3; k++) {
      side_upto[k].assign(1, 0);
      blk_upto[k].assign(1, 0);
    }
    for (int q = 0; q < n; q++) {
      Engine<T> *e = members[q].e;
      if (e->p.num_td || e->p.num_fd) {
        GroupSide<T> it{};
        it.kind = 0;
        it.td_pts = e->d_td_pts;
        it.num_td = e->p.num_td;
        it.fd_pts = e->d_fd_pts;
        it.num_fd = e->p.num_fd;
        it.td_buf = e->d_td;
        it.fd_stage = e->d_stage;
        it.out_start = e->p.out_start;
        it.out_stop = e->out_last();
        it.tblock = kStageRows;
        items[0].push_back(it);
        owner[0].push_back(q);
      }
      for (const SrcLaunch &l : e->srcs) {
        GroupSide<T> it{};
        it.kind = 1;
        it.b = l.b;
        it.c = l.c;
        it.skind = l.kind;
        it.soft = (T)l.soft;
        it.values = (const T *)l.values;
        const int k = l.c <= EZ ? 1 : 2;
        items[k].push_back(it);
        owner[k].push_back(q);
      }
    }
    size_t o_side[3];
    for (int k = 0; k < 3; k++) o_side[k] = place(sizeof(GroupSide<T>) * items[k].size());
    const size_t o_grids = place(sizeof(Grid<T>) * (size_t)n);
    const size_t o_steps = place(sizeof(uint64_t *) * (size_t)n);
    const size_t total = off;
    char *dbase = nullptr;
    if (da.alloc(&dbase, total)) return VGPU_ENOMEM;
    CK(cudaHostAlloc((void **)&host, total, cudaHostAllocDefault));
    memset(host, 0, total);
    d_err = (int *)(dbase + o_err);
    counters = (int *)(dbase + o_counters);
    for (int h = 0; h < 2; h++)
      for (int c = 0; c < 2; c++) {
        GroupMesh<T> *gm = (GroupMesh<T> *)(host + o_mesh[h][c]);
        GroupTile *gt = (GroupTile *)(host + o_tiles[h][c]);
        int nt = 0;
        for (int q = 0; q < n; q++) {
          const int r = cls_index[h][c][q];
          if (r < 0) continue;
          Engine<T> *e = members[q].e;
          const auto &L = (h == 0 ? e->sw_e : e->sw_h)[c];
          GroupMesh<T> &M = gm[r];
          M.maps = h == 0 ? e->maps_e : e->maps_h;
          for (int a = 0; a < 3; a++) M.mc.F[a] = e->g.F[(h == 0 ? EX : HX) + a];
          const PmlFull<T> &pf = h == 0 ? e->pfe : e->pfh;
          for (int a = 0; a < 6; a++) M.mc.aux[a] = pf.aux[a];
          M.mc.s0 = e->g.s0;
          M.mc.s1 = e->g.s1;
          M.mc.n1 = e->g.n1;
          M.mc.wn = M.maps.wn;
          M.headers = L.headers;
          const CoefIndex &ci = h == 0 ? e->cie : e->cih;
          M.table = (const T *)(dbase + o_tab[2 * q + h]);
          M.tab_bytes = (uint32_t)(((size_t)ci.ntab * (h == 0 ? 6 : 3) * sizeof(T) + 15) / 16 * 16);
          const size_t hb = c ? sizeof(SweepHeader<T, true>) : sizeof(SweepHeader<T, false>);
          for (int u = 0; u < L.ntiles; u++)
            gt[nt++] = GroupTile{ L.host[u], r, (const char *)L.headers + hb * (size_t)u, M.table, M.tab_bytes,
                                  M.mc.wn };
        }
        meshes[h][c] = (GroupMesh<T> *)(dbase + o_mesh[h][c]);
        tiles[h][c] = (GroupTile *)(dbase + o_tiles[h][c]);
      }
    Grid<T> *grids_d = (Grid<T> *)(dbase + o_grids);
    Grid<T> *grids_h = (Grid<T> *)(host + o_grids);
    uint64_t **steps_h = (uint64_t **)(host + o_steps);
    for (int q = 0; q < n; q++) {
      grids_h[q] = members[q].e->g;
      steps_h[q] = members[q].e->d_step;
    }
    for (int k = 0; k < 3; k++) {
      GroupSide<T> *it = (GroupSide<T> *)(host + o_side[k]);
      int blk = 0;
      size_t r = 0;
      for (int q = 0; q < n; q++) {
        for (; r < items[k].size() && owner[k][r] == q; r++) {
          GroupSide<T> x = items[k][r];
          x.g = grids_d + q;
          x.step = members[q].e->d_step;
          const int64_t pts = x.kind == 0 ? (int64_t)(x.num_td + x.num_fd) * 6 : x.b.count();
          x.first_block = blk;
          blk += (int)Engine<T>::blocks_for(pts, 128);
          it[r] = x;
        }
        side_upto[k].push_back((int)r);
        blk_upto[k].push_back(blk);
      }
      side[k] = (GroupSide<T> *)(dbase + o_side[k]);
    }
    steps = (uint64_t **)(dbase + o_steps);
    CK(cudaMemcpyAsync(dbase, host, total, cudaMemcpyHostToDevice, s));
    for (int q = 0; q < n; q++)
      for (int h = 0; h < 2; h++) {
        const CoefIndex &ci = h == 0 ? members[q].e->cie : members[q].e->cih;
        CK(cudaMemcpyAsync(dbase + o_tab[2 * q + h], ci.table, (size_t)ci.ntab * (h == 0 ? 6 : 3) * sizeof(T),
                           cudaMemcpyDeviceToDevice, s));
      }
    if (int rc = new_view()) return rc;
    CK(cudaEventRecord(t0, s));
    return 0;
  }

  // Graphs for the first R members (captured on first use); the previous
  // view is released once its launches have run.
  int new_view()
  {
    if (cur) {
      CK(cudaEventRecord(cur->done, s));
      retired.push_back(cur);
      cur = nullptr;
      rebuilds++;
    }
    for (size_t q = 0; q < retired.size();) {
      if (cudaEventQuery(retired[q]->done) == cudaSuccess) {
        release(retired[q]);
        retired.erase(retired.begin() + (long)q);
      } else {
        cudaGetLastError();
        q++;
      }
    }
    if (!R) return 0;
    View *v = new View();
    cur = v;
    v->R = R;
    CK(cudaEventCreateWithFlags(&v->done, cudaEventDisableTiming));
    for (int h = 0; h < 2; h++)
      for (int c = 0; c < 2; c++) {
        const int nt = tiles_upto[h][c][R];
        v->ntiles[h][c] = nt;
        v->grid[h][c] = (int)std::min<int64_t>((nt + chunk - 1) / chunk, (int64_t)per_sm[h][c] * nsm);
      }
    return 0;
  }

  template <bool ES, bool PML>
  void launch_sweep(const View &v, int h, int c, int rel)
  {
    static const SweepMaps kNoMaps{};
    k_sweep_tma<T, ES, PML, true><<<v.grid[h][c], kSweepThreads, SweepLayout<T, ES, PML>::smem_bytes(true), s>>>(
        kNoMaps, Grid<T>{}, nullptr, nullptr, v.ntiles[h][c], PmlFull<T>{}, CoefIndex{}, d_err, meshes[h][c],
        tiles[h][c], counters + rel * 4 + h * 2 + c, chunk);
  }

  // One step's launches for the view's members, `rel` steps past their
  // counters.
  uint64_t enqueue_step(const View &v, int rel)
  {
    const int r = v.R;
    uint64_t n = 0;
    auto side_launch = [&](int k) {
      if (!side_upto[k][r]) return;
      k_group_side<T><<<blk_upto[k][r], 128, 0, s>>>(side[k], side_upto[k][r], rel);
      n++;
    };
    auto sweep = [&](int h, int c) {
      if (!v.grid[h][c]) return;
      if (h == 0 && c == 0) launch_sweep<true, false>(v, 0, 0, rel);
      if (h == 0 && c == 1) launch_sweep<true, true>(v, 0, 1, rel);
      if (h == 1 && c == 0) launch_sweep<false, false>(v, 1, 0, rel);
      if (h == 1 && c == 1) launch_sweep<false, true>(v, 1, 1, rel);
      n++;
    };
    side_launch(0);
    sweep(0, 0);
    sweep(0, 1);
    side_launch(1);
    sweep(1, 0);
    sweep(1, 1);
    side_launch(2);
    return n;
  }

  int capture(View &v, int q)
  {
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int len = kGraphSteps >> q;
    uint64_t n = 0;
    // Every sweep launch of the graph takes its tiles from its own counter.
    cudaMemsetAsync(counters, 0, sizeof(int) * 4 * len, s);
    for (int rel = 0; rel < len; rel++) n = enqueue_step(v, rel);
    k_group_advance<<<Engine<T>::blocks_for(v.R, 128), 128, 0, s>>>(steps, v.R, len);
    v.per_step = n;
    const cudaError_t ee = cudaStreamEndCapture(s, &gr);
    if (ee != cudaSuccess) return set_err(VGPU_ECUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ee));
    const cudaError_t e = cudaGraphInstantiate(&v.graphs[q], gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
      v.graphs[q] = nullptr;
      return set_err(VGPU_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    }
    return 0;
  }

  // The next block: up to the next 64-step boundary and no member past its
  // count; then each member's own block-end work (DFT fold, energy check)
  // on the group's stream, and a new view when members have finished.
  int issue_block() override
  {
    // Members sit at the same step modulo the block length; the last active
    // member has the fewest steps left.
    uint64_t m = std::min<uint64_t>(kChunk - (members[0].e->step % kChunk), members[R - 1].left);
    const uint64_t block = m;
    for (int q = 0; q < 5 && m; q++) {
      const uint64_t len = (uint64_t)(kGraphSteps >> q);
      while (m >= len) {
        if (!cur->graphs[q])
          if (int rc = capture(*cur, q)) return rc;
        CK(cudaGraphLaunch(cur->graphs[q], s));
        launches += len * cur->per_step + 1;
        m -= len;
      }
    }
    for (int q = 0; q < R; q++) {
      Member &mb = members[q];
      Engine<T> *e = mb.e;
      const uint64_t n0 = e->step;
      mb.left -= block;
      e->stats.steps += block;
      const cudaStream_t own = e->s;
      e->s = s;
      const uint64_t before = e->stats.kernel_launches;
      const int rc = e->after_block(n0, block, (int)((n0 / kChunk) & 1));
      launches += e->stats.kernel_launches - before;
      e->s = own;
      if (rc) return rc;
    }
    const int r0 = R;
    while (R > 0 && members[R - 1].left == 0) R--;
    if (R != r0)
      if (int rc = new_view()) return rc;
    return 0;
  }

  // Wait for the group's work; a pipeline failure is handed to every
  // member (its later launches skip, and it reports VGPU_ETIMEOUT).
  int finish() override
  {
    if (!s || !d_err) return 0;
    CK(cudaEventRecord(t1, s));
    CK(cudaStreamSynchronize(s));
    float t = 0;
    if (cudaEventElapsedTime(&t, t0, t1) == cudaSuccess) ms = t;
    int h = 0;
    CK(cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    int rc = 0;
    std::string msg;
    for (Engine<T> *e : all) {
      if (h) CK(cudaMemcpy(e->d_err, &h, sizeof(int), cudaMemcpyHostToDevice));
      e->stats.run_ms = ms;
      if (int r = e->finish_queued())
        if (!rc) {
          rc = r;
          msg = g_err;
        }
    }
    if (rc) set_err(rc, "%s", msg.c_str());
    return rc;
  }
};

struct vgpu_engine {
  EngineBase *impl;
  int dev;   // the CUDA device the engine was created on
};

// The engine's implementation, with its device made current on the calling
// thread: engines may be driven from threads other than the creating one.
static EngineBase *on_dev(const vgpu_engine *e)
{
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != e->dev) cudaSetDevice(e->dev);
  return e->impl;
}

static int validate(const vgpu_problem *p)
{
  if (!p) return set_err(VGPU_EINVAL, "null problem");
  if (p->abi_version != VGPU_ABI_VERSION) return set_err(VGPU_EINVAL, "ABI version %d, expected %d", p->abi_version, VGPU_ABI_VERSION);
  if (p->precision != VGPU_FP64 && p->precision != VGPU_FP32) return set_err(VGPU_EINVAL, "invalid precision %d", p->precision);
  for (int a = 0; a < 3; a++)
    if (p->n[a] < 3) return set_err(VGPU_EINVAL, "grid extent n[%d]=%d too small", a, p->n[a]);
  for (int q = 0; q < 9; q++)
    if (!p->coef[q]) return set_err(VGPU_EINVAL, "coefficient volume %d missing", q);
  for (int a = 0; a < 3; a++)
    if (!p->ide[a] || !p->idh[a]) return set_err(VGPU_EINVAL, "edge length arrays missing");
  // Every limit used by an update must keep its stencil inside the volume:
  // E updates read the -1 neighbours, H updates the +1 neighbours.
  // Only the two axes other than the component's own are offset.
  auto in_grid = [&](const int32_t l[6], int field) {
    if (l[1] < l[0] || l[3] < l[2] || l[5] < l[4]) return true;
    for (int a = 0; a < 3; a++) {
      bool reach = a != field % 3;
      int lo = (field <= 2 && reach) ? 1 : 0, hi_off = (field > 2 && reach) ? 2 : 1;
      if (l[2 * a] < lo || l[2 * a + 1] > p->n[a] - hi_off) return false;
    }
    return true;
  };
  for (int f = 0; f < 6; f++)
    if (!in_grid(p->gfilim[f], f)) return set_err(VGPU_EINVAL, "bulk limits of field %d outside the grid", f);
  for (int r = 0; r < 6; r++)
    if (p->pml_present[r])
      for (int f = 0; f < 6; f++)
        if (!in_grid(p->pml_flim[r][f], f)) return set_err(VGPU_EINVAL, "PML limits outside the grid");
  for (int q = 0; q < p->num_sources; q++) {
    const int32_t *l = p->sources[q].flim;
    if (!(l[1] < l[0] || l[3] < l[2] || l[5] < l[4]) &&
        (l[0] < 0 || l[2] < 0 || l[4] < 0 || l[1] >= p->n[0] || l[3] >= p->n[1] || l[5] >= p->n[2]))
      return set_err(VGPU_EINVAL, "source %d limits outside the grid", q);
    if (p->num_steps && !p->sources[q].values) return set_err(VGPU_EINVAL, "source %d has no values", q);
  }
  for (int q = 0; q < p->num_td; q++)
    for (int a = 0; a < 3; a++)
      if (p->td_points[3 * q + a] < 0 || p->td_points[3 * q + a] >= p->n[a]) return set_err(VGPU_EINVAL, "observer point outside the grid");
  for (int q = 0; q < p->num_fd; q++)
    for (int a = 0; a < 3; a++)
      if (p->fd_points[3 * q + a] < 0 || p->fd_points[3 * q + a] >= p->n[a]) return set_err(VGPU_EINVAL, "observer point outside the grid");
  return 0;
}

extern "C" int vgpu_create(const vgpu_problem *p, vgpu_engine **out)
{
  if (!out) return set_err(VGPU_EINVAL, "null output pointer");
  *out = nullptr;
  if (int rc = validate(p)) return rc;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return set_err(VGPU_ENODEV, "no CUDA device: %s", cudaGetErrorString(e));
  int dev = 0;
  cudaGetDevice(&dev);
  // Two attributes, not cudaGetDeviceProperties, which queries every
  // property and costs milliseconds per engine.
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (major != 10) return set_err(VGPU_ENODEV, "device %d is sm_%d%d; this engine is built for sm_100a", dev, major, minor);
  EngineBase *impl = nullptr;
  int rc;
  if (p->precision == VGPU_FP64) {
    auto *en = new Engine<double>();
    rc = en->create(p);
    impl = en;
  } else {
    auto *en = new Engine<float>();
    rc = en->create(p);
    impl = en;
  }
  if (rc) {
    delete impl;
    return rc;
  }
  *out = new vgpu_engine{ impl, dev };
  return 0;
}

// Host-only check of the sweep plan: each swept component's bulk and UPML
// points are claimed by exactly one tile and no other point is; tiles keep
// the kernel's limits (planes, k alignment, narrow auxiliary boxes that
// cover the UPML points of their tile).
extern "C" int vgpu_check_sweep_plan(const vgpu_problem *p, int32_t precision, int64_t *violations, int64_t *tiles)
{
  if (!p || !violations || !tiles) return set_err(VGPU_EINVAL, "null argument");
  if (int rc = validate(p)) return rc;
  const int halo = precision == VGPU_FP64 ? 2 : 4;
  const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
  const RegionSet rs = regions_of(*p);
  int64_t bad = 0, ntiles = 0;
  std::vector<uint8_t> claims((size_t)n0 * n1 * n2);
  for (int es = 0; es < 2; es++) {
    Box bb[3];
    for (int c = 0; c < 3; c++) bb[c] = box_from(p->gfilim[(es ? 0 : 3) + c]);
    if (!es) fold_mur_h(*p, bb);
    const SweepPlan pl = plan_sweep(unite(bb), rs, es != 0, halo, 148, g_tune_depth);
    std::vector<SweepTile> all(pl.bulk);
    all.insert(all.end(), pl.pml.begin(), pl.pml.end());
    ntiles += (int64_t)all.size();
    for (const SweepTile &t : all) {
      if (t.i1 - t.i0 + 1 > kSweepMaxPlanes || t.i1 < t.i0 || t.k0 % kSweepKW) bad++;
      if (t.ax >= 0 && (t.ax % halo || pl.wn <= 0)) bad++;
    }
    for (int c = 0; c < 3; c++) {
      const int f = (es ? EX : HX) + c;
      std::fill(claims.begin(), claims.end(), 0);
      for (const SweepTile &t : all) {
        const Box tb = tile_box(t);
        for (int i = std::max(tb.i0, 0); i <= std::min(tb.i1, n0 - 1); i++)
          for (int j = std::max(tb.j0, 0); j <= std::min(tb.j1, n1 - 1); j++)
            for (int k = std::max(tb.k0, 0); k <= std::min(tb.k1, n2 - 1); k++) {
              int n = (t.bulk && bb[c].contains(i, j, k)) ? 1 : 0;
              for (int r = 0; r < 2; r++) {
                if (t.reg[r] < 0 || !rs.lim[t.reg[r]][f].contains(i, j, k)) continue;
                n++;
                if (t.ax >= 0 && (k < t.ax || k >= t.ax + pl.wn)) bad++;   // auxiliaries not loaded
              }
              uint8_t &cl = claims[((size_t)i * n1 + j) * n2 + k];
              cl = (uint8_t)std::min(255, cl + n);
            }
      }
      for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
          for (int k = 0; k < n2; k++) {
            int want = bb[c].contains(i, j, k) ? 1 : 0;
            for (int q = 0; q < rs.nreg; q++) want += rs.lim[q][f].contains(i, j, k) ? 1 : 0;
            if (want > 1) want = -1;   // overlapping boxes: the engine refuses such problems
            if (want >= 0 && claims[((size_t)i * n1 + j) * n2 + k] != want) bad++;
          }
    }
  }
  *violations = bad;
  *tiles = ntiles;
  return 0;
}

extern "C" int vgpu_set_device(int32_t device)
{
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return set_err(VGPU_ENODEV, "cudaSetDevice(%d): %s", (int)device, cudaGetErrorString(e));
  return 0;
}

extern "C" int vgpu_get_device(int32_t *device)
{
  if (!device) return set_err(VGPU_EINVAL, "null argument");
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) return set_err(VGPU_ENODEV, "cudaGetDevice: %s", cudaGetErrorString(e));
  *device = d;
  return 0;
}

extern "C" int vgpu_run(vgpu_engine *e, uint64_t nsteps)
{
  if (!e) return set_err(VGPU_EINVAL, "null engine");
  return on_dev(e)->run(nsteps);
}

extern "C" int vgpu_read_td(vgpu_engine *e, double *out, uint64_t steps)
{
  if (!e || !out) return set_err(VGPU_EINVAL, "null argument");
  return on_dev(e)->read_td(out, steps);
}

extern "C" int vgpu_read_dft(vgpu_engine *e, double *re, double *im)
{
  if (!e || !re || !im) return set_err(VGPU_EINVAL, "null argument");
  return on_dev(e)->read_dft(re, im);
}

extern "C" int vgpu_read_field(vgpu_engine *e, int32_t c, double *out)
{
  if (!e || !out || c < 0 || c > 5) return set_err(VGPU_EINVAL, "invalid argument");
  return on_dev(e)->read_field(c, out);
}

extern "C" int vgpu_write_field(vgpu_engine *e, int32_t c, const double *in)
{
  if (!e || !in || c < 0 || c > 5) return set_err(VGPU_EINVAL, "invalid argument");
  return on_dev(e)->write_field(c, in);
}

extern "C" int vgpu_check_finite(vgpu_engine *e)
{
  if (!e) return set_err(VGPU_EINVAL, "null engine");
  return on_dev(e)->check_finite();
}

extern "C" uint64_t vgpu_current_step(const vgpu_engine *e) { return e ? e->impl->step : 0; }

extern "C" int vgpu_enqueue(vgpu_engine *e, uint64_t max_steps, uint64_t *queued)
{
  if (!e || !queued) return set_err(VGPU_EINVAL, "null argument");
  return on_dev(e)->enqueue(max_steps, queued);
}

extern "C" int vgpu_query(vgpu_engine *e)
{
  if (!e) return set_err(VGPU_EINVAL, "null engine");
  return on_dev(e)->query();
}

extern "C" int vgpu_synchronize(vgpu_engine *e)
{
  if (!e) return set_err(VGPU_EINVAL, "null engine");
  return on_dev(e)->synchronize();
}

extern "C" int vgpu_run_batch(vgpu_engine *const *engines, int32_t n, const uint64_t *steps)
{
  if (n < 0 || (n && (!engines || !steps))) return set_err(VGPU_EINVAL, "invalid batch");
  for (int32_t i = 0; i < n; i++) {
    if (!engines[i]) return set_err(VGPU_EINVAL, "null engine %d in batch", (int)i);
    if (int rc = on_dev(engines[i])->check_steps(steps[i])) return rc;
  }
  std::vector<uint64_t> left(steps, steps + n);
  // On a queueing error nothing more is queued, but every engine's queued
  // blocks are still waited for: the caller gets control back only when no
  // engine of the batch is stepping.  The first error is returned.
  int rc = 0;
  std::string msg;
  for (bool any = true; any && !rc;) {
    any = false;
    for (int32_t i = 0; i < n && !rc; i++) {
      if (!left[i]) continue;
      uint64_t m = 0;
      if (int r = on_dev(engines[i])->enqueue(left[i], &m)) {
        rc = r;
      } else if (!m) {
        // An engine listed twice can reach its last step before its count.
        rc = set_err(VGPU_EINVAL, "engine %d in batch reached its last step", (int)i);
      }
      if (rc) msg = g_err;
      left[i] -= m;
      any = any || left[i] > 0;
    }
  }
  for (int32_t i = 0; i < n; i++) {
    int r = on_dev(engines[i])->synchronize();
    if (r && !rc) {
      rc = r;
      msg = g_err;
    }
  }
  if (rc) set_err(rc, "%s", msg.c_str());
  return rc;
}

extern "C" void *vgpu_host_alloc(uint64_t bytes) { return host_blocks().alloc((size_t)bytes); }

extern "C" void vgpu_host_free(void *ptr)
{
  if (ptr) host_blocks().release(ptr);
}

extern "C" int vgpu_set_sweep_tuning(int32_t march_depth, int32_t blocks_per_sm, int32_t group_chunk)
{
  if (march_depth < 0 || march_depth > kSweepMaxPlanes || blocks_per_sm < 0 || group_chunk < 0 || group_chunk > 4096)
    return set_err(VGPU_EINVAL, "sweep tuning: march depth 0..%d, blocks per SM >= 0, group chunk 0..4096",
                   kSweepMaxPlanes);
  g_tune_depth = march_depth;
  g_tune_blocks = blocks_per_sm;
  g_tune_chunk = group_chunk;
  return 0;
}

extern "C" int vgpu_groupable(const vgpu_engine *e)
{
  if (!e) return set_err(VGPU_EINVAL, "null engine");
  EngineBase *b = on_dev(e);
  if (auto *f = dynamic_cast<Engine<float> *>(b)) return f->groupable() ? 1 : 0;
  if (auto *d = dynamic_cast<Engine<double> *>(b)) return d->groupable() ? 1 : 0;
  return 0;
}

// Members of one precision's group: groupable engines on the first engine's
// device at a 64-step boundary, after their earlier work has finished.
template <typename T>
static int collect(Group<T> &G, vgpu_engine *const *engines, int32_t n, const uint64_t *steps, std::vector<char> &taken)
{
  for (int32_t i = 0; i < n; i++) {
    if (!steps[i] || taken[i] || engines[i]->dev != engines[0]->dev) continue;
    auto *e = dynamic_cast<Engine<T> *>(on_dev(engines[i]));
    if (!e || !e->groupable() || e->step % kChunk) continue;
    if (int rc = e->synchronize()) return rc;
    G.members.push_back({ e, steps[i] });
    taken[i] = 1;
  }
  // One engine alone gains nothing from a group.
  if (G.members.size() == 1) {
    for (int32_t i = 0; i < n; i++)
      if (engines[i]->impl == G.members[0].e) taken[i] = 0;
    G.members.clear();
  }
  return 0;
}

extern "C" int vgpu_run_grouped(vgpu_engine *const *engines, int32_t n, const uint64_t *steps,
                                vgpu_group_report *report)
{
  if (report) memset(report, 0, sizeof *report);
  if (n < 0 || (n && (!engines || !steps))) return set_err(VGPU_EINVAL, "invalid batch");
  for (int32_t i = 0; i < n; i++) {
    if (!engines[i]) return set_err(VGPU_EINVAL, "null engine %d in batch", (int)i);
    for (int32_t k = 0; k < i; k++)
      if (engines[k] == engines[i]) return set_err(VGPU_EINVAL, "engine %d listed twice in batch", (int)i);
    if (int rc = on_dev(engines[i])->check_steps(steps[i])) return rc;
  }
  if (!n) return 0;
  std::vector<char> taken((size_t)n, 0);
  Group<float> g32;
  Group<double> g64;
  if (int rc = collect(g32, engines, n, steps, taken)) return rc;
  if (int rc = collect(g64, engines, n, steps, taken)) return rc;
  GroupBase *groups[2] = { &g32, &g64 };
  std::vector<uint64_t> left((size_t)n, 0), before((size_t)n, 0);
  for (int32_t i = 0; i < n; i++)
    if (!taken[i]) {
      left[i] = steps[i];
      before[i] = on_dev(engines[i])->stats.kernel_launches;
    }
  // As vgpu_run_batch: on an error nothing more is queued, everything queued
  // is waited for, and the first error is returned.
  int rc = 0;
  std::string msg;
  auto fail = [&](int r) {
    if (r && !rc) {
      rc = r;
      msg = g_err;
    }
  };
  cudaSetDevice(engines[0]->dev);
  if (!g32.members.empty()) fail(g32.start());
  if (!rc && !g64.members.empty()) fail(g64.start());
  for (bool any = true; any && !rc;) {
    any = false;
    for (GroupBase *g : groups)
      if (!rc && g->busy()) {
        cudaSetDevice(engines[0]->dev);
        fail(g->issue_block());
        any = any || g->busy();
      }
    for (int32_t i = 0; i < n && !rc; i++) {
      if (!left[i]) continue;
      uint64_t m = 0;
      int r = on_dev(engines[i])->enqueue(left[i], &m);
      if (!r && !m) r = set_err(VGPU_EINVAL, "engine %d in batch reached its last step", (int)i);
      fail(r);
      left[i] -= m;
      any = any || left[i] > 0;
    }
  }
  for (GroupBase *g : groups) {
    cudaSetDevice(engines[0]->dev);
    fail(g->finish());
  }
  uint64_t launches = g32.launches + g64.launches;
  for (int32_t i = 0; i < n; i++)
    if (!taken[i]) {
      fail(on_dev(engines[i])->synchronize());
      launches += on_dev(engines[i])->stats.kernel_launches - before[i];
    }
  if (report) {
    report->launches = launches;
    report->grouped = g32.members_at_start + g64.members_at_start;
    report->rebuilds = g32.rebuilds + g64.rebuilds;
    report->tiles = g32.tiles_at_start + g64.tiles_at_start;
    report->group_ms = std::max(g32.ms, g64.ms);
  }
  if (rc) set_err(rc, "%s", msg.c_str());
  return rc;
}

extern "C" int vgpu_sweep_points(const vgpu_engine *e, int32_t kernel, uint64_t *bulk_points, uint64_t *pml_points)
{
  if (!e || !bulk_points || !pml_points) return set_err(VGPU_EINVAL, "null argument");
  return on_dev(e)->sweep_points(kernel, bulk_points, pml_points);
}

extern "C" int vgpu_set_bin_sink(vgpu_engine *e, vgpu_bin_sink sink, void *user)
{
  if (!e) return set_err(VGPU_EINVAL, "null engine");
  on_dev(e)->bin_sink = sink;
  on_dev(e)->bin_user = user;
  return 0;
}

extern "C" int vgpu_time_kernel(vgpu_engine *e, int32_t kernel, int32_t warmup, int32_t iters, double *ms,
                                uint64_t *points)
{
  if (!e || !ms || !points || iters < 0 || warmup < 0) return set_err(VGPU_EINVAL, "invalid argument");
  return on_dev(e)->time_kernel(kernel, warmup, iters, ms, points);
}

extern "C" int vgpu_get_stats(const vgpu_engine *e, vgpu_stats *st)
{
  if (!e || !st) return set_err(VGPU_EINVAL, "null argument");
  *st = on_dev(e)->stats;
  return 0;
}

extern "C" int vgpu_set_sweep_wait_limit(int64_t polls)
{
  const uint32_t v = polls < 0 ? kSpinLimit : (uint32_t)std::min<int64_t>(polls, kSpinLimit);
  CK(cudaMemcpyToSymbol(g_full_wait_polls, &v, sizeof v));
  return 0;
}

// ---------------------------------------------------------------------------
// Allocation-free running DFT for callers that cannot allocate device
// memory.  The twiddle table lives in a file-scope device array; every GPU
// that loads this library holds it (1 MiB) until the process exits.
// ---------------------------------------------------------------------------

static __device__ __align__(256) double2 g_static_twiddle[VGPU_STATIC_DFT_MAX_ENTRIES];
static std::mutex g_static_mu;
static double2 *g_static_twiddle_ptr[64];  // device address of g_static_twiddle, per device

extern "C" int vgpu_dft_accumulate_static(const double *samples, int32_t num_series, int32_t num_rows,
                                          const double *omega, int32_t num_freq, double dt, uint64_t first_step,
                                          double *re, double *im)
{
  if (!samples || !omega || !re || !im) return set_err(VGPU_EINVAL, "null device pointer");
  if (num_series <= 0 || num_rows <= 0 || num_freq <= 0) return set_err(VGPU_EINVAL, "sizes must be positive");
  if (num_rows > VGPU_STATIC_DFT_MAX_ROWS)
    return set_err(VGPU_EINVAL, "num_rows %d exceeds the maximum of %d rows per call", num_rows, VGPU_STATIC_DFT_MAX_ROWS);
  if (num_series > VGPU_STATIC_DFT_MAX_SERIES)
    return set_err(VGPU_EINVAL, "num_series %d exceeds the maximum of %d series per call", num_series,
                   VGPU_STATIC_DFT_MAX_SERIES);
  if ((int64_t)num_rows * num_freq > VGPU_STATIC_DFT_MAX_ENTRIES)
    return set_err(VGPU_EINVAL, "num_rows * num_freq = %lld exceeds the static twiddle table of %d entries",
                   (long long)num_rows * num_freq, VGPU_STATIC_DFT_MAX_ENTRIES);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_err(VGPU_EINVAL, "device ordinal %d out of range", dev);
  double2 *tw = nullptr;
  {
    // First call on a device: look up the array's device address with that
    // device current.  Host code may not use the symbol itself as a pointer.
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_twiddle_ptr[dev]) {
      void *ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_twiddle);
      if (e != cudaSuccess) return set_err(VGPU_ECUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      g_static_twiddle_ptr[dev] = (double2 *)ptr;
    }
    tw = g_static_twiddle_ptr[dev];
  }
  // The table is fully rewritten for the rows of this call before it is read,
  // so nothing needs clearing; re/im carry the running sums between calls.
  int64_t ntw = (int64_t)num_rows * num_freq;
  k_twiddle<<<(unsigned)((ntw + 127) / 128), 128, 0, 0>>>(omega, num_freq, dt, first_step, 0, num_rows, tw);
  dim3 blk(32, 8), grd((num_freq + 31) / 32, (num_series + 7) / 8);
  k_dft_accumulate<<<grd, blk, sizeof(double) * 8 * num_rows, 0>>>(samples, num_series, num_freq, num_rows, 0,
                                                                  num_rows, tw, re, im);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(0));
  return 0;
}

extern "C" void vgpu_destroy(vgpu_engine *e)
{
  if (!e) return;
  delete on_dev(e);
  delete e;
}
