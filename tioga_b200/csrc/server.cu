// Serving form: a request loop over many resident overset systems.
//
// Each request is one time step of one system: rigid motions of some of its
// blocks, then preprocess, connectivity and (optionally) the data update, the
// reference's per-step call sequence (src/tiogaInterface.C:150-216) for that
// system alone.  Systems stay resident between their requests (their
// engine: topology, cell trees, hole-map slabs, donor rest state and
// coordinates on the device; a step refits the tree boxes to the moved
// coordinates instead of rebuilding the trees).
//
// Scheduling is continuous: `nslots` workers take requests in arrival order
// as soon as a slot is free, so requests that arrive while others run are
// admitted at once and their kernels overlap on the GPU (every engine has its
// own stream).  A system is made resident when it fits the HBM budget (its
// bytes measured by the engine's own allocations, estimated before its first
// step); otherwise idle resident systems without pending requests are
// evicted, least recently used first (their device coordinates are written
// back to the caller's arrays first), and a request that still does not fit
// waits.  Requests of one system run one at a time and in order, so each
// result is the one the system would get alone.
//
// Device buffers come stream-ordered from the server's own memory pool,
// reserved up front to the budget (less what the device has free).  Growing
// a pool maps new memory under a lock that every allocating thread waits for
// (30-70 ms per growth on B200), so a pool that grew whenever a moving mesh
// pushed a buffer past its last size stalled every slot at once; the
// reserved pool serves those growths from memory it already holds.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace tb {

namespace {
double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace

// request statuses besides 0 (success) and the engine's own error codes
constexpr int kSrvOverBudget = -3;  // the system alone needs more than the HBM budget
constexpr int kSrvCancelled = -4;   // cancelled before it started
constexpr int kSrvTimedOut = -5;    // a bounded wait ended first (the request goes on)

struct SrvBlock {
  int tag, nnodes, ncells, nwbc, nobc, ntypes;
  double* x;
  int* ibl;
  int* wbc;
  int* obc;
  int nv[4], nc[4];
  int* conn[4];
};

struct SrvRequest {
  long long ticket = 0;
  int sys = 0;
  std::vector<int> move_tag;
  std::vector<double> moves;  // 12 per move: a (row-major 3x3), b
  int nvar = 0;
  std::vector<double*> q;     // per block, or empty (no data update)
  bool q_device = false;      // q points to device arrays (a GPU solver's fields)
  std::vector<int*> ibl;      // per block iblank destination, or empty (the registered arrays)
  double t_submit = 0, t_start = 0, t_done = 0;
  double t_pre = 0, t_conn = 0, t_upd = 0;  // host time of the three calls
  long long nquery = 0, nreceptor = 0, nhole = 0;
  int rc = 0;
  bool done = false;
};

struct SrvSystem {
  std::vector<SrvBlock> blocks;
  Engine* eng = nullptr;
  long long bytes = 0;       // device bytes held (resident) or reserved (being admitted)
  long long last_bytes = 0;  // bytes when it was last resident
  bool busy = false;         // a request (or its eviction) is running
  double last_used = 0;
  int pending = 0;           // queued requests
};

class Server {
 public:
  Server(long long budget, int nslots, int max_resident)
      : budget_(budget), nslots_(std::max(1, nslots)), max_resident_(std::max(1, max_resident)) {
    cudaGetDevice(&device_);
    make_pool();
    for (int i = 0; i < nslots_; i++) workers_.emplace_back([this] { work(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : workers_) t.join();
    for (auto& kv : sys_) {
      if (kv.second.eng) {
        g_dbuf_stream = kv.second.eng->stream();
        delete kv.second.eng;
        g_dbuf_stream = nullptr;
      }
    }
    for (auto& kv : req_) delete kv.second;
    if (pool_) {  // its memory goes back to the device once the frees above complete
      cudaDeviceSynchronize();
      cudaMemPoolDestroy(pool_);
    }
  }

  int add_block(int sys, const SrvBlock& b) {
    std::lock_guard<std::mutex> g(mu_);
    SrvSystem& S = sys_[sys];
    if (S.eng || S.busy || S.pending) {
      fprintf(stderr, "#tioga_b200: server: blocks are added before a system's first request\n");
      return -1;
    }
    for (const SrvBlock& o : S.blocks)
      if (o.tag == b.tag) {
        fprintf(stderr, "#tioga_b200: server: system %d already has mesh tag %d\n", sys, b.tag);
        return -1;
      }
    S.blocks.push_back(b);
    return 0;
  }

  long long submit(SrvRequest* r) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = sys_.find(r->sys);
    if (it == sys_.end() || it->second.blocks.empty()) {
      fprintf(stderr, "#tioga_b200: server: unknown system %d\n", r->sys);
      delete r;
      return -1;
    }
    const size_t nb = it->second.blocks.size();
    if ((!r->q.empty() && r->q.size() != nb) || (!r->ibl.empty() && r->ibl.size() != nb)) {
      delete r;
      return -1;
    }
    r->ticket = next_ticket_++;
    r->t_submit = now_ms();
    it->second.pending++;
    queue_.push_back(r);
    req_[r->ticket] = r;
    cv_work_.notify_one();
    return r->ticket;
  }

  // Blocks until the request is done, or for at most timeout_ms when that is
  // >= 0: kSrvTimedOut then, and the ticket stays valid for a later wait.
  int wait(long long ticket, double times[6], long long counts[4], double timeout_ms = -1.0) {
    std::unique_lock<std::mutex> l(mu_);
    auto it = req_.find(ticket);
    if (it == req_.end()) return -1;
    SrvRequest* r = it->second;
    if (timeout_ms < 0) {
      cv_done_.wait(l, [&] { return r->done; });
    } else if (!cv_done_.wait_for(l, std::chrono::duration<double, std::milli>(timeout_ms), [&] { return r->done; })) {
      return kSrvTimedOut;
    }
    if (times) {
      times[0] = r->t_done - r->t_submit;
      times[1] = r->t_start - r->t_submit;
      times[2] = r->t_done - r->t_start;
      times[3] = r->t_pre;
      times[4] = r->t_conn;
      times[5] = r->t_upd;
    }
    if (counts) {
      counts[0] = r->nquery;
      counts[1] = r->nreceptor;
      counts[2] = r->nhole;
      counts[3] = r->rc;
    }
    const int rc = r->rc;
    req_.erase(it);
    delete r;
    return rc;
  }

  // A request that has not started is taken out of the queue and completes
  // with kSrvCancelled; one that runs or has finished cannot be cancelled.
  int cancel(long long ticket) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = req_.find(ticket);
    if (it == req_.end()) return -1;
    SrvRequest* r = it->second;
    auto q = std::find(queue_.begin(), queue_.end(), r);
    if (q == queue_.end()) return -1;
    queue_.erase(q);
    sys_[r->sys].pending--;
    finish_unrun(r, kSrvCancelled);
    return 0;
  }

  int nblocks(int sys) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = sys_.find(sys);
    return it == sys_.end() ? -1 : (int)it->second.blocks.size();
  }

  void stats(long long out[16]) {
    std::lock_guard<std::mutex> g(mu_);
    for (int i = 0; i < 16; i++) out[i] = 0;
    int res = 0;
    for (auto& kv : sys_) res += kv.second.eng ? 1 : 0;
    out[0] = res;
    out[1] = used_;
    out[2] = admissions_;
    out[3] = evictions_;
    out[4] = completed_;
    out[5] = (long long)queue_.size();
    out[6] = budget_;
    out[7] = peak_used_;
    out[8] = reserved_;
    cudaMemPool_t pool = pool_;
    if (!pool) cudaDeviceGetDefaultMemPool(&pool, device_);
    unsigned long long v = 0;
    if (pool && cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v) == cudaSuccess)
      out[9] = (long long)v;
  }

 private:
  // bytes a system needs before it has been resident once: per node, per
  // cell and per hole-map slab, with headroom
  static long long estimate(const SrvSystem& S) {
    long long n = 0, c = 0, w = 0;
    for (const SrvBlock& b : S.blocks) {
      n += b.nnodes;
      c += b.ncells;
      w += b.nwbc > 0;
    }
    return 320 * n + 320 * c + (long long)kHoleMapCap * w + (16ll << 20);
  }

  // under the lock: the first queued request that can run now, with the
  // systems to evict for it (marked busy)
  SrvRequest* pick(std::vector<int>& evict) {
    std::map<int, bool> blocked;  // a system whose earlier request waits keeps its order
    for (auto it = queue_.begin(); it != queue_.end(); ++it) {
      SrvRequest* r = *it;
      if (blocked.count(r->sys)) continue;
      SrvSystem& S = sys_[r->sys];
      if (S.busy) {
        blocked[r->sys] = true;
        continue;
      }
      if (!S.eng) {
        // a system larger than the whole budget is refused (kSrvOverBudget)
        const long long need = S.last_bytes > 0 ? S.last_bytes : estimate(S);
        if (need > budget_) {
          fprintf(stderr, "#tioga_b200: server: system %d needs %lld bytes, over the budget of %lld\n", r->sys,
                  need, budget_);
          queue_.erase(it);
          S.pending--;
          finish_unrun(r, kSrvOverBudget);
          return pick(evict);
        }
        int res = 0;
        for (auto& kv : sys_) res += (kv.second.eng != nullptr || kv.second.bytes > 0) ? 1 : 0;
        long long freed = 0;
        std::vector<std::pair<double, int>> idle;
        for (auto& kv : sys_)
          if (kv.second.eng && !kv.second.busy && kv.second.pending == 0)
            idle.push_back({kv.second.last_used, kv.first});
        std::sort(idle.begin(), idle.end());
        std::vector<int> ev;
        size_t k = 0;
        while ((used_ - freed + need > budget_ || res - (int)ev.size() + 1 > max_resident_) && k < idle.size()) {
          ev.push_back(idle[k].second);
          freed += sys_[idle[k].second].bytes;
          k++;
        }
        if (used_ - freed + need > budget_ || res - (int)ev.size() + 1 > max_resident_) {
          blocked[r->sys] = true;  // waits for memory
          continue;
        }
        for (int e : ev) sys_[e].busy = true;
        evict = ev;
        S.bytes = need;  // reserved until its engine reports its own bytes
        used_ += need;
        admissions_++;
      }
      S.busy = true;
      S.pending--;
      queue_.erase(it);
      return r;
    }
    return nullptr;
  }

  // under the lock: a request that will not run completes with status rc
  void finish_unrun(SrvRequest* r, int rc) {
    r->rc = rc;
    r->t_start = r->t_done = now_ms();
    r->done = true;
    cv_done_.notify_all();
  }

  // The server's pool: freed buffers stay in it for the next allocation, and
  // min(budget, free device memory - 2 GiB) is reserved at once by one
  // allocation freed at the end of its stream.  Without a pool of its own
  // (creation failed) the device's default pool is used the same way.
  void make_pool() {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    if (cudaMemPoolCreate(&pool_, &props) != cudaSuccess) {
      cudaGetLastError();
      pool_ = nullptr;
      if (cudaDeviceGetDefaultMemPool(&def_pool_, device_) != cudaSuccess) def_pool_ = nullptr;
    }
    cudaMemPool_t pool = pool_ ? pool_ : def_pool_;
    if (!pool) return;
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    const long long want = std::min(budget_, (long long)free_b - (2ll << 30)) & ~((2ll << 20) - 1);
    if (want < (64ll << 20)) return;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, (size_t)want, pool, s) == cudaSuccess) {
      cudaFreeAsync(p, s);
      reserved_ = want;
    } else {
      cudaGetLastError();  // no reservation: the pool grows on demand
    }
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }

  void work() {
    cudaSetDevice(device_);
    g_dbuf_pool = pool_;  // null: cudaMallocAsync from the default pool
    std::unique_lock<std::mutex> l(mu_);
    for (;;) {
      std::vector<int> evict;
      SrvRequest* r = nullptr;
      while (!stop_ && !(r = pick(evict))) cv_work_.wait(l);
      if (stop_ && !r) return;
      l.unlock();
      for (int e : evict) {  // write the coordinates back, free the device memory
        SrvSystem& E = sys_.at(e);
        g_dbuf_account = &E.bytes;
        g_dbuf_stream = E.eng->stream();
        E.eng->download_coords();
        delete E.eng;
        g_dbuf_account = nullptr;
        g_dbuf_stream = nullptr;
        l.lock();
        used_ -= E.last_bytes;  // what it held at its last step
        E.bytes = 0;
        E.eng = nullptr;
        E.busy = false;
        evictions_++;
        l.unlock();
      }
      SrvSystem& S = sys_.at(r->sys);
      r->t_start = now_ms();
      run(S, r);
      r->t_done = now_ms();
      l.lock();
      if (S.eng) {
        used_ += S.eng->device_bytes() - S.bytes;
        S.bytes = S.eng->device_bytes();
        S.last_bytes = S.bytes;
      } else {
        used_ -= S.bytes;
        S.bytes = 0;
      }
      peak_used_ = std::max(peak_used_, used_);
      S.busy = false;
      S.last_used = r->t_done;
      r->done = true;
      completed_++;
      cv_done_.notify_all();
      cv_work_.notify_all();
    }
  }

  void run(SrvSystem& S, SrvRequest* r) {
    int rc = 0;
    bool fresh = false;
    if (!S.eng) {  // admission: the system's engine, its topology and coordinates
      Engine* e = new Engine();
      {  // published under the lock: pick() and stats() read the pointer
        std::lock_guard<std::mutex> g(mu_);
        S.eng = e;
      }
      g_dbuf_account = S.eng->byte_counter();
      g_dbuf_stream = S.eng->stream();
      for (const SrvBlock& b : S.blocks) {
        rc = S.eng->register_block(b.tag, b.nnodes, b.x, b.ibl, b.nwbc, b.nobc, b.wbc, b.obc, b.ntypes, b.nv, b.nc,
                                   const_cast<int**>(b.conn));
        if (rc) break;
      }
      S.eng->set_coords_resident(1);
      S.eng->set_serving(true);
      fresh = true;
    }
    Engine& E = *S.eng;
    g_dbuf_account = E.byte_counter();
    g_dbuf_stream = E.stream();
    if (!rc && fresh && !r->move_tag.empty()) rc = E.preprocess();  // coordinates on the device first
    for (size_t m = 0; !rc && m < r->move_tag.size(); m++) {
      const int b = E.find_block(0, r->move_tag[m]);
      rc = (b < 0) ? -1 : E.apply_rigid(b, &r->moves[12 * m], &r->moves[12 * m + 9]);
    }
    for (size_t b = 0; b < S.blocks.size(); b++) E.set_host_iblank((int)b, r->ibl.empty() ? S.blocks[b].ibl : r->ibl[b]);
    double t = now_ms();
    if (!rc) rc = E.preprocess();
    r->t_pre = now_ms() - t;
    t = now_ms();
    if (!rc) rc = E.connectivity();
    r->t_conn = now_ms() - t;
    t = now_ms();
    if (!rc && !r->q.empty()) {
      for (size_t b = 0; b < S.blocks.size() && !rc; b++)
        rc = E.register_solution(S.blocks[b].tag, r->q[b], r->q_device);
      if (!rc) rc = E.dataupdate(r->nvar, 0);
    }
    r->t_upd = now_ms() - t;
    const Stats& st = E.stats();
    r->nquery = st.nquery;
    r->nreceptor = st.nreceptor;
    r->nhole = st.nhole;
    r->rc = rc ? rc : (st.error ? -(int)st.error : 0);
    g_dbuf_account = nullptr;
    g_dbuf_stream = nullptr;
  }

  long long budget_;
  int nslots_, max_resident_;
  int device_ = 0;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::map<int, SrvSystem> sys_;
  std::deque<SrvRequest*> queue_;
  std::map<long long, SrvRequest*> req_;
  long long next_ticket_ = 1, used_ = 0, peak_used_ = 0, admissions_ = 0, evictions_ = 0, completed_ = 0;
  bool stop_ = false;
  cudaMemPool_t pool_ = nullptr, def_pool_ = nullptr;
  long long reserved_ = 0;  // bytes reserved in the pool at creation
  std::vector<std::thread> workers_;
};

}  // namespace tb

#pragma GCC visibility push(default)
#include "../../include/tioga_b200.h"

extern "C" {

void* tioga_b200_server_create(long long hbm_budget_bytes, int nslots, int max_resident) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    fprintf(stderr, "#tioga_b200: no CUDA device; the serving form cannot run\n");
    return nullptr;
  }
  return new tb::Server(hbm_budget_bytes, nslots, max_resident);
}

void tioga_b200_server_destroy(void* srv) { delete static_cast<tb::Server*>(srv); }

int tioga_b200_server_add_block(void* srv, int sys, int btag, int nnodes, double* xyz, int* ibl, int nwbc, int nobc,
                                int* wbcnode, int* obcnode, int ntypes, const int* nv, const int* nc,
                                int* const* vconn) {
  if (!srv || ntypes < 1 || ntypes > 4) return -1;
  tb::SrvBlock b{};
  b.tag = btag;
  b.nnodes = nnodes;
  b.x = xyz;
  b.ibl = ibl;
  b.nwbc = nwbc;
  b.nobc = nobc;
  b.wbc = wbcnode;
  b.obc = obcnode;
  b.ntypes = ntypes;
  b.ncells = 0;
  for (int t = 0; t < 4; t++) {
    b.nv[t] = t < ntypes ? nv[t] : 0;
    b.nc[t] = t < ntypes ? nc[t] : 0;
    b.conn[t] = t < ntypes ? vconn[t] : nullptr;
    b.ncells += b.nc[t];
  }
  return static_cast<tb::Server*>(srv)->add_block(sys, b);
}

long long tioga_b200_server_submit(void* srv, int sys, int nmoves, const int* move_tags, const double* moves,
                                   int nvar, double* const* q, int* const* ibl_out) {
  return tioga_b200_server_submit_fields(srv, sys, nmoves, move_tags, moves, nvar, q, 0, ibl_out);
}

long long tioga_b200_server_submit_fields(void* srv, int sys, int nmoves, const int* move_tags, const double* moves,
                                          int nvar, double* const* q, int q_on_device, int* const* ibl_out) {
  if (!srv || nmoves < 0 || (nmoves > 0 && (!move_tags || !moves))) return -1;
  auto* r = new tb::SrvRequest();
  r->q_device = q_on_device != 0;
  r->sys = sys;
  r->move_tag.assign(move_tags, move_tags + nmoves);
  r->moves.assign(moves, moves + 12 * (size_t)nmoves);
  r->nvar = nvar;
  auto* s = static_cast<tb::Server*>(srv);
  // per-block pointer lists: their length is the system's block count,
  // which the server checks
  if (q || ibl_out) {
    const int nb = s->nblocks(sys);
    if (nb <= 0) {
      delete r;
      return -1;
    }
    if (q) r->q.assign(q, q + nb);
    if (ibl_out) r->ibl.assign(ibl_out, ibl_out + nb);
  }
  return s->submit(r);
}

int tioga_b200_server_wait(void* srv, long long ticket, double times_ms[6], long long counts[4]) {
  if (!srv) return -1;
  return static_cast<tb::Server*>(srv)->wait(ticket, times_ms, counts);
}

int tioga_b200_server_wait_timeout(void* srv, long long ticket, double timeout_ms, double times_ms[6],
                                   long long counts[4]) {
  if (!srv) return -1;
  return static_cast<tb::Server*>(srv)->wait(ticket, times_ms, counts, timeout_ms < 0 ? 0.0 : timeout_ms);
}

int tioga_b200_server_cancel(void* srv, long long ticket) {
  if (!srv) return -1;
  return static_cast<tb::Server*>(srv)->cancel(ticket);
}

void tioga_b200_server_stats(void* srv, long long out[16]) {
  if (!srv) {
    for (int i = 0; i < 16; i++) out[i] = 0;
    return;
  }
  static_cast<tb::Server*>(srv)->stats(out);
}

}  // extern "C"

#pragma GCC visibility pop
