// msc_batch_solve: many slab solves of uneven size, frequency and incidence on one
// GPU.
//
// Small slabs cannot fill a B200 on their own (an Arnoldi step of a 16 x 16 x 4
// slab is a few microseconds of launches on a few dozen SMs), so the batch runs
// several solves at once: `workers` host threads each own a stream, a small cache
// of plans (LRU, keyed by geometry and background) and pinned staging buffers, and
// take items from a shared counter. Every plan's work runs on its own stream, so the
// solves of different workers overlap on the device; their GMRES cycles run
// uncaptured (a graph capture per new plan costs more than a short solve saves).
// Plan memory comes from the library's memory pool, so the plan churn of a batch over
// many shapes reuses device memory instead of mapping it again. A solved field leaves
// the device by DMA into one of the worker's two page-locked buffers; a copier thread
// moves it into the caller's array while the workers carry on. With workers = 0 an
// online autotuner times the first items at 1, 2 and 4 workers and finishes the batch
// with the fastest, and the lateral FFT length of each aperiodic shape is autotuned (the
// smallest 2,3,5,7-smooth length or the next power of two, timed once per shape:
// msc_slab_desc.Lxy = -1). Items are independent: a failed item records its status and the
// others continue.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "plan.cuh"

namespace msc {

namespace {

constexpr int BATCH_PLANS_PER_WORKER = 2;

struct CachedPlan {
  msc_slab_desc key;
  msc_plan* plan = nullptr;
  long long last_use = 0;
};

// Page-locked host staging of one batch worker: the contrasts of an item on their way
// in, and two buffers for fields on their way out. Kept per (device, worker index)
// for the life of the process, grown to the largest item seen, so later batch calls
// pay no cudaHostAlloc.
struct PinnedStaging {
  void* in = nullptr;
  size_t in_bytes = 0;
  void* out[2] = {nullptr, nullptr};
  size_t out_bytes[2] = {0, 0};
};

PinnedStaging& pinned_staging(int device, int worker) {
  static std::mutex mu;
  static std::vector<std::vector<PinnedStaging*>> all;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)all.size() <= device) all.resize(device + 1);
  auto& v = all[device];
  while ((int)v.size() <= worker) v.push_back(new PinnedStaging());
  return *v[worker];
}

int grow_pinned(void*& p, size_t& have, size_t need) {
  if (have >= need) return MSC_OK;
  if (p) cudaFreeHost(p);
  p = nullptr;
  have = 0;
  if (cudaMallocHost(&p, need) != cudaSuccess) {
    cudaGetLastError();
    set_error("batch: pinned staging of %zu bytes failed", need);
    return MSC_ERR_NOMEM;
  }
  have = need;
  return MSC_OK;
}

// Moves fields from the workers' pinned buffers into the callers' arrays on its own
// host thread, so the host copy of one item overlaps the device work of the next ones.
struct Copier {
  struct Job {
    cudaEvent_t ev;
    const void* src;
    void* dst;
    size_t bytes;
    std::atomic<int>* busy;
  };
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job> q;
  bool stop = false;
  std::atomic<bool> failed{false};
  std::thread th;

  explicit Copier(int device) {
    th = std::thread([this, device]() {
      cudaSetDevice(device);
      while (true) {
        Job j;
        {
          std::unique_lock<std::mutex> lk(mu);
          cv.wait(lk, [&] { return stop || !q.empty(); });
          if (q.empty()) return;
          j = q.front();
          q.pop_front();
        }
        if (cudaEventSynchronize(j.ev) != cudaSuccess) failed.store(true);
        else std::memcpy(j.dst, j.src, j.bytes);
        j.busy->store(0);
      }
    });
  }
  void push(const Job& j) {
    {
      std::lock_guard<std::mutex> lk(mu);
      q.push_back(j);
    }
    cv.notify_one();
  }
  // drains the queue and ends the thread
  void finish() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_one();
    if (th.joinable()) th.join();
  }
  ~Copier() { finish(); }
};

struct Worker {
  bool tune_fft = false;  // workers = 0: the lateral FFT length of aperiodic plans is autotuned
  cudaStream_t stream = nullptr;
  int device = 0;
  int index = 0;
  std::vector<CachedPlan> plans;
  long long tick = 0;
  // device staging: contrasts (3 N float64), psi0 and x (9 N complex128 each)
  void* dev = nullptr;
  size_t dev_bytes = 0;
  PinnedStaging* pin = nullptr;
  // fields in flight to the caller: copied into pin->out[s] on the stream (event ev[s]),
  // then into the caller's array by the copier; busy[s] until the copier is done
  Copier* copier = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  std::atomic<int> busy[2];
  int slot = 0;

  Worker() {
    busy[0] = 0;
    busy[1] = 0;
  }
  Worker(const Worker&) = delete;
  Worker& operator=(const Worker&) = delete;
  ~Worker() {
    drain();
    for (auto& c : plans)
      if (c.plan) msc_plan_destroy(c.plan);
    if (dev) cudaFreeAsync(dev, stream);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }

  int init(int dev_index, int worker_index, Copier* c) {
    device = dev_index;
    index = worker_index;
    copier = c;
    pin = &pinned_staging(dev_index, worker_index);
    MSC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (auto& e : ev) MSC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return MSC_OK;
  }

  void wait_slot(int s) {
    while (busy[s].load()) std::this_thread::yield();
  }
  // every field of this worker has reached its caller's array
  void drain() {
    wait_slot(0);
    wait_slot(1);
  }

  // queue the device field x (bytes) for the caller's host array h
  int send(void* h, const void* x, size_t bytes) {
    const int s = slot;
    slot ^= 1;
    wait_slot(s);
    MSC_TRY(grow_pinned(pin->out[s], pin->out_bytes[s], bytes));
    MSC_CUDA(cudaMemcpyAsync(pin->out[s], x, bytes, cudaMemcpyDeviceToHost, stream));
    MSC_CUDA(cudaEventRecord(ev[s], stream));
    busy[s].store(1);
    copier->push(Copier::Job{ev[s], pin->out[s], h, bytes, &busy[s]});
    return MSC_OK;
  }

  int plan_for(const msc_slab_desc& d, msc_plan** out) {
    ++tick;
    for (auto& c : plans)
      if (std::memcmp(&c.key, &d, sizeof(d)) == 0) {
        c.last_use = tick;
        *out = c.plan;
        return MSC_OK;
      }
    if ((int)plans.size() >= BATCH_PLANS_PER_WORKER) {
      auto it = std::min_element(plans.begin(), plans.end(),
                                 [](const CachedPlan& a, const CachedPlan& b) { return a.last_use < b.last_use; });
      msc_plan_destroy(it->plan);
      plans.erase(it);
    }
    msc_plan* p = nullptr;
    msc_slab_desc dd = d;
    if (tune_fft && !dd.periodic && dd.Lxy == 0) dd.Lxy = -1;  // autotuned lateral FFT length
    const int s = msc_plan_create(&dd, stream, &p);
    if (s != MSC_OK) return s;
    // a batch item is one short solve on a plan that is rarely reused: capturing and
    // instantiating its GMRES cycles costs more than it saves
    p->graphs = false;
    CachedPlan c;
    std::memcpy(&c.key, &d, sizeof(d));
    c.plan = p;
    c.last_use = tick;
    plans.push_back(c);
    *out = p;
    return MSC_OK;
  }

  int staging(size_t dbytes, size_t hbytes) {
    if (dev_bytes < dbytes) {
      if (dev) cudaFreeAsync(dev, stream);
      dev = nullptr;
      dev_bytes = 0;
      if (pool_alloc(&dev, dbytes, device, stream) != cudaSuccess) {
        cudaGetLastError();
        set_error("batch: device staging of %zu bytes failed", dbytes);
        return MSC_ERR_NOMEM;
      }
      dev_bytes = dbytes;
    }
    if (pin->in_bytes < hbytes) {
      cudaStreamSynchronize(stream);
      MSC_TRY(grow_pinned(pin->in, pin->in_bytes, hbytes));
    }
    return MSC_OK;
  }

  // One item end to end; its statistics and R_PP are written in place.
  int solve(msc_batch_item& it, const msc_solve_opts& o) {
    msc_plan* pl = nullptr;
    MSC_TRY(plan_for(it.desc, &pl));
    const size_t ns = (size_t)it.desc.N_z * it.desc.M * it.desc.M;
    const size_t fb = sizeof(double2) * 9 * ns;
    MSC_TRY(staging(3 * sizeof(double) * ns + 2 * fb, 3 * sizeof(double) * ns));
    double* dc = (double*)dev;
    double2* psi0 = (double2*)(dc + 3 * ns);
    double2* x = psi0 + 9 * ns;
    double* hc = (double*)pin->in;
    MSC_CUDA(cudaStreamSynchronize(stream));  // the pinned buffer is free again
    std::memcpy(hc, it.dlam, sizeof(double) * ns);
    std::memcpy(hc + ns, it.dmu, sizeof(double) * ns);
    std::memcpy(hc + 2 * ns, it.drho, sizeof(double) * ns);
    MSC_CUDA(cudaMemcpyAsync(dc, hc, 3 * sizeof(double) * ns, cudaMemcpyHostToDevice, stream));
    MSC_TRY(msc_build_t0(pl, dc, dc + ns, dc + 2 * ns, it.omega));
    const double nk = std::sqrt(it.k_hat[0] * it.k_hat[0] + it.k_hat[1] * it.k_hat[1] + it.k_hat[2] * it.k_hat[2]);
    const double speed = it.wave_type == MSC_WAVE_P ? it.desc.alpha : it.desc.beta;
    double kpar[2] = {0.0, 0.0};
    if (it.bloch) {
      kpar[0] = it.omega / speed * it.k_hat[1] / nk;
      kpar[1] = it.omega / speed * it.k_hat[2] / nk;
    }
    MSC_TRY(msc_build_g0(pl, it.omega, it.bloch ? kpar : nullptr, it.volume_averaged ? 1 : 0,
                         it.n_orders > 0 ? it.n_orders : 2));
    MSC_TRY(msc_incident(pl, it.omega, it.k_hat, it.wave_type, psi0));
    msc_solve_stats st{};
    const int s = msc_solve(pl, psi0, x, &o, &st);
    it.stats = st;
    if (s < 0) return s;
    // specular R_PP: at the item's slowness, by default the horizontal slowness of the
    // incidence for Bloch items, else normal incidence (the reference's default)
    const double p = it.rpp_p >= 0 ? it.rpp_p
                     : it.bloch ? std::sqrt(it.k_hat[1] * it.k_hat[1] + it.k_hat[2] * it.k_hat[2]) / nk / speed
                                : 0.0;
    MSC_TRY(msc_rpp_periodic(pl, x, it.omega, p, it.bloch ? MSC_RPP_BLOCH : 0, it.rpp));
    // the field: a DMA into a pinned buffer on the stream; the host moves it into the
    // caller's (pageable) array while the worker's next item runs on the device
    if (it.psi) MSC_TRY(send(it.psi, x, fb));
    return s;
  }
};

// Solve items [next, end) with w workers; returns the elapsed seconds.
double run_workers(std::vector<Worker>& pool, int w, msc_batch_item* items, std::atomic<int>& next, int end,
                   const msc_solve_opts& o, int device) {
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  for (int i = 0; i < w; ++i) {
    th.emplace_back([&, i]() {
      cudaSetDevice(device);
      Worker& wk = pool[i];
      while (true) {
        // claim the next item below `end` without moving the counter past it, so the
        // items after a chunk stay for the next chunk
        int k = next.load();
        while (k < end && !next.compare_exchange_weak(k, k + 1)) {
        }
        if (k >= end) break;
        msc_batch_item& it = items[k];
        const int s = wk.solve(it, o);
        it.status = s;
        if (s < 0) {
          std::strncpy(it.error, msc_last_error(), sizeof(it.error) - 1);
          it.error[sizeof(it.error) - 1] = 0;
        }
      }
      // the fields still in flight reach the caller before the chunk counts as done
      wk.drain();
    });
  }
  for (auto& t : th) t.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace msc

using namespace msc;

extern "C" int msc_batch_solve(msc_batch_item* items, int n, const msc_solve_opts* opts, int workers,
                               int* workers_used) {
  if ((!items && n > 0) || !opts || n < 0) {
    set_error("null argument");
    return MSC_ERR_INVALID;
  }
  if (workers < 0 || workers > 64) {
    set_error("workers must be in [0, 64], got %d", workers);
    return MSC_ERR_INVALID;
  }
  for (int i = 0; i < n; ++i) {
    msc_batch_item& it = items[i];
    if (!it.dlam || !it.dmu || !it.drho) {
      set_error("item %d: null contrast array", i);
      return MSC_ERR_INVALID;
    }
    it.status = MSC_NOT_CONVERGED;
    it.error[0] = 0;
    it.rpp[0] = it.rpp[1] = 0.0;
    std::memset(&it.stats, 0, sizeof(it.stats));
  }
  int device = 0;
  MSC_CUDA(cudaGetDevice(&device));
  const int maxw = workers > 0 ? workers : 4;
  Copier copier(device);
  std::vector<Worker> pool(maxw);
  for (int i = 0; i < maxw; ++i) {
    MSC_TRY(pool[i].init(device, i, &copier));
    pool[i].tune_fft = workers == 0;
  }
  std::atomic<int> next{0};
  int chosen = workers;
  if (workers == 0) {
    // online autotune: chunks of items at 1, 2 and 4 workers, time per item compared;
    // the search stops at the first count that is slower than the best so far (more
    // threads contend for the driver as well as the device)
    const int chunk = std::max(2, std::min(16, n / 8));
    double best = 1e300;
    chosen = 1;
    for (int w : {1, 2, 4}) {
      const int start = next.load();
      if (start >= n) break;
      const int end = std::min(n, start + std::max(1, chunk * w / 2));
      const double t = run_workers(pool, w, items, next, end, *opts, device);
      const double per = t / std::max(1, end - start);
      if (per >= best) break;
      best = per;
      chosen = w;
    }
  }
  if (next.load() < n) run_workers(pool, chosen, items, next, n, *opts, device);
  copier.finish();
  if (copier.failed.load()) {
    set_error("batch: a field's copy to the host failed");
    return MSC_ERR_CUDA;
  }
  if (workers_used) *workers_used = chosen;
  for (int i = 0; i < n; ++i)
    if (items[i].status != MSC_OK) return MSC_NOT_CONVERGED;
  return MSC_OK;
}
