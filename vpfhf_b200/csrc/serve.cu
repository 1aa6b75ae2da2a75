// serve.cu -- the request loop: independent fracture problems on one GPU, admitted
// in arrival order as workers and device memory free up, each solved on a pooled
// ctx of its grid size, overlapping on the device through the contexts' streams.
//
// Host code only.  A worker thread takes the oldest queued request, acquires a ctx
// (an idle pooled ctx of the same grid; else a new one if the memory estimate fits
// the budget; else the least recently used idle ctx of another grid is destroyed
// and the admission retried; else it waits for a running problem to finish), runs
// the problem through the public C ABI and returns the ctx to the pool.  A pooled
// ctx keeps its solver work space and captured CG graphs; the per-problem
// parameters live in device memory that the graphs read, so reuse is exact.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "abi_util.h"
#include "vec.h"

using namespace vfgpu;
using clk = std::chrono::steady_clock;

namespace {

// A pooled ctx serves problems of one grid and one multigrid mode (mg: 0 = Jacobi U
// solve, else the V-cycle's bytes per value), so that its reservation covers the
// hierarchy it holds.
struct GridKey {
  int nx, ny, nz;
  double lx, ly, lz;
  int mg;
  bool operator==(const GridKey& o) const {
    return nx == o.nx && ny == o.ny && nz == o.nz && lx == o.lx && ly == o.ly && lz == o.lz &&
           mg == o.mg;
  }
};

struct Slot {
  vfgpu_ctx* ctx;
  GridKey key;
  long long bytes;
  bool busy;
  uint64_t last_used;
};

struct Job {
  unsigned long long ticket;
  vfgpu_request req;
  double t_submit;
};

}  // namespace

struct vfgpu_server {
  int dev = 0;
  long long budget = 0, reserved = 0, peak_reserved = 0;
  int nworkers = 0, contexts_created = 0, evictions = 0;
  long long submitted = 0, completed = 0, running = 0;
  int freeing = 0;  // evicted contexts being destroyed (their bytes still reserved)
  unsigned long long next_ticket = 1;
  uint64_t use_counter = 0;
  bool stop = false;
  clk::time_point t0 = clk::now();
  std::mutex m;
  std::condition_variable cv_job, cv_done, cv_mem;
  std::deque<Job> queue;
  std::deque<vfgpu_result> done;
  std::vector<Slot> pool;
  std::vector<std::thread> workers;

  double now() const { return std::chrono::duration<double>(clk::now() - t0).count(); }
};

namespace {

GridKey key_of(const vfgpu_request& q) {
  const vfgpu_grid& g = q.grid;
  const int pc = resolve_pc(q.opts.pc, g.nx, g.ny, g.nz);
  const int mg = pc == VFGPU_PC_MG ? (q.opts.precision == VFGPU_MIXED ? 4 : 8) : 0;
  return {g.nx, g.ny, g.nz, g.lx, g.ly, g.lz, mg};
}

// Takes an idle ctx of the job's grid or makes room for a new one.  Called with the
// lock held; may release it while destroying or creating contexts.  Returns the pool
// index of the acquired slot (and counts the job in `running`), or -1 with `rc` and
// `err` set.  A job waits for memory only while some other job is running: when none
// is, nothing will free memory and the job fails with VFGPU_ERR_OOM.
int acquire(vfgpu_server* s, std::unique_lock<std::mutex>& lk, const GridKey& key, bool* reused,
            int* rc, std::string* err) {
  vfgpu_grid g{key.nx, key.ny, key.nz, key.lx, key.ly, key.lz};
  long long need = 0;
  if (vfgpu_memory_estimate(&g, &need) != VFGPU_OK) {
    *rc = VFGPU_ERR_INVALID;
    *err = vfgpu_last_error();
    return -1;
  }
  if (key.mg) need += mg_memory_bytes(key.nx, key.ny, key.nz, key.mg);
  auto oom = [&] {
    *rc = VFGPU_ERR_OOM;
    char b[160];
    std::snprintf(b, sizeof b, "serving: a %dx%dx%d problem needs %lld bytes, budget %lld",
                  key.nx, key.ny, key.nz, need, s->budget);
    *err = b;
    return -1;
  };
  if (need > s->budget) return oom();
  for (;;) {
    for (size_t i = 0; i < s->pool.size(); i++)
      if (!s->pool[i].busy && s->pool[i].key == key) {
        s->pool[i].busy = true;
        s->running++;
        *reused = true;
        return (int)i;
      }
    if (s->reserved + need <= s->budget) {
      s->reserved += need;
      s->peak_reserved = std::max(s->peak_reserved, s->reserved);
      s->running++;  // counts from the reservation on, so that waiters see progress coming
      lk.unlock();
      vfgpu_ctx* c = nullptr;
      const int r = vfgpu_create(&g, &c);
      const std::string msg = r ? vfgpu_last_error() : "";
      lk.lock();
      if (r != VFGPU_OK) {
        s->reserved -= need;
        s->running--;
        s->cv_mem.notify_all();
        *rc = r;
        *err = msg;
        return -1;
      }
      s->contexts_created++;
      s->pool.push_back({c, key, need, true, 0});
      *reused = false;
      return (int)s->pool.size() - 1;
    }
    // evict the least recently used idle ctx (of another grid: an idle ctx of this
    // grid would have been taken above)
    int victim = -1;
    for (size_t i = 0; i < s->pool.size(); i++)
      if (!s->pool[i].busy && (victim < 0 || s->pool[i].last_used < s->pool[victim].last_used))
        victim = (int)i;
    if (victim >= 0) {
      Slot v = s->pool[victim];
      s->pool.erase(s->pool.begin() + victim);
      s->evictions++;
      s->freeing++;
      lk.unlock();
      vfgpu_destroy(v.ctx);
      lk.lock();
      s->reserved -= v.bytes;
      s->freeing--;
      s->cv_mem.notify_all();
      continue;
    }
    if (s->running == 0 && s->freeing == 0) return oom();  // nothing will free memory
    s->cv_mem.wait(lk);
  }
}

// The problem itself, through the public ABI on a ctx of the right grid.
int solve(vfgpu_ctx* c, const vfgpu_request& q, vfgpu_result* r) {
  int rc;
  if ((rc = vfgpu_set_matprop(c, 1, &q.mp, nullptr))) return rc;
  if ((rc = vfgpu_set_cell_modulus(c, nullptr))) return rc;
  if ((rc = vfgpu_set_vfprop(c, &q.vf))) return rc;
  if ((rc = vfgpu_set_bc(c, q.bcU, &q.bcV))) return rc;
  // VFFieldsInitialize defaults (U = BCU = theta = thetaRef = 0) and the pressure
  cudaError_t e = cudaSuccess;
  const int zero[] = {VFGPU_FIELD_U, VFGPU_FIELD_BCU, VFGPU_FIELD_THETA, VFGPU_FIELD_THETAREF};
  for (int f : zero)
    if (e == cudaSuccess) e = fill_f64(c->f[f], 0.0, field_len(c, f), c->stream);
  if (e == cudaSuccess) e = fill_f64(c->f[VFGPU_FIELD_PRESSURE], q.pressure, c->N, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "serving: field initialisation");
  if ((rc = vfgpu_init_cracks(c, q.npenny, q.penny, q.nrect, q.rect))) return rc;
  if ((rc = vfgpu_time_step_prepare(c))) return rc;
  const int maxit = q.am_its > 0 ? q.am_its : q.max_am_its;
  for (int it = 0; it < maxit; it++) {
    vfgpu_solve_stats su{}, sv{};
    double err = 0;
    rc = vfgpu_am_step(c, &q.opts, &err, &su, &sv);
    if (rc < 0) return rc;
    r->am_its = it + 1;
    r->am_err = err;
    r->ksp_its_u += su.ksp_its;
    r->ksp_its_v += sv.ksp_its;
    if (q.am_its <= 0 && err < q.altmintol) break;
  }
  double insitu = 0;
  if ((rc = vfgpu_u_energy(c, &r->elastic, &insitu, &r->pressure_work))) return rc;
  if ((rc = vfgpu_v_energy(c, &r->surface))) return rc;
  if ((rc = vfgpu_crack_opening(c, &r->cov, q.out_cellcov))) return rc;
  if (q.out_u && (rc = vfgpu_get_field(c, VFGPU_FIELD_U, q.out_u))) return rc;
  if (q.out_v && (rc = vfgpu_get_field(c, VFGPU_FIELD_V, q.out_v))) return rc;
  return VFGPU_OK;
}

void worker_main(vfgpu_server* s, int wid) {
  cudaSetDevice(s->dev);
  std::unique_lock<std::mutex> lk(s->m);
  for (;;) {
    s->cv_job.wait(lk, [&] { return s->stop || !s->queue.empty(); });
    if (s->queue.empty()) return;  // stop requested and nothing left
    Job job = s->queue.front();
    s->queue.pop_front();
    vfgpu_result r{};
    r.ticket = job.ticket;
    r.tag = job.req.tag;
    r.t_submit = job.t_submit;
    r.worker = wid;
    bool reused = false;
    std::string err;
    int rc = VFGPU_OK;
    const int slot = acquire(s, lk, key_of(job.req), &reused, &rc, &err);
    if (slot >= 0) {
      vfgpu_ctx* c = s->pool[slot].ctx;
      lk.unlock();
      r.t_start = s->now();
      r.reused_ctx = reused;
      rc = solve(c, job.req, &r);
      if (rc != VFGPU_OK && rc != VFGPU_NOT_CONVERGED && rc != VFGPU_DIVERGED) err = vfgpu_last_error();
      r.t_done = s->now();
      lk.lock();
      s->running--;
      // the slot index may have moved (evictions erase entries): find the ctx again
      for (auto& sl : s->pool)
        if (sl.ctx == c) {
          sl.busy = false;
          sl.last_used = ++s->use_counter;
        }
      s->cv_mem.notify_all();
    } else {
      r.t_start = r.t_done = s->now();
    }
    r.status = rc;
    std::snprintf(r.error, sizeof r.error, "%s", err.c_str());
    s->completed++;
    s->done.push_back(r);
    s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int vfgpu_server_create(int device, int workers, long long budget_bytes, vfgpu_server** out) {
  if (!out || workers < 1 || workers > 256)
    return fail(VFGPU_ERR_INVALID, "vfgpu_server_create: need 1..256 workers");
  cudaError_t e = cudaSetDevice(device);
  size_t fr = 0, tot = 0;
  if (e == cudaSuccess) e = cudaMemGetInfo(&fr, &tot);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_server_create");
  auto* s = new vfgpu_server;
  s->dev = device;
  s->budget = budget_bytes > 0 ? budget_bytes : (long long)(0.85 * (double)fr);
  s->nworkers = workers;
  for (int w = 0; w < workers; w++) s->workers.emplace_back(worker_main, s, w);
  *out = s;
  return VFGPU_OK;
}

int vfgpu_server_submit(vfgpu_server* s, const vfgpu_request* q, unsigned long long* ticket) {
  if (!s || !q) return fail(VFGPU_ERR_INVALID, "vfgpu_server_submit: null argument");
  if (q->grid.nx < 2 || q->grid.ny < 2 || q->grid.nz < 2 || !(q->grid.lx > 0) ||
      !(q->grid.ly > 0) || !(q->grid.lz > 0))
    return fail(VFGPU_ERR_INVALID, "vfgpu_server_submit: bad grid");
  if (q->npenny < 0 || q->npenny > VFGPU_SERVE_MAX_PENNY || q->nrect < 0 ||
      q->nrect > VFGPU_SERVE_MAX_RECT)
    return fail(VFGPU_ERR_INVALID, "vfgpu_server_submit: at most %d penny and %d rectangular cracks",
                VFGPU_SERVE_MAX_PENNY, VFGPU_SERVE_MAX_RECT);
  if (q->am_its <= 0 && q->max_am_its <= 0)
    return fail(VFGPU_ERR_INVALID, "vfgpu_server_submit: need am_its > 0 or max_am_its > 0");
  std::lock_guard<std::mutex> lk(s->m);
  if (s->stop) return fail(VFGPU_ERR_STATE, "vfgpu_server_submit: server is stopping");
  Job j{s->next_ticket++, *q, s->now()};
  if (ticket) *ticket = j.ticket;
  s->queue.push_back(j);
  s->submitted++;
  s->cv_job.notify_one();
  return VFGPU_OK;
}

int vfgpu_server_next(vfgpu_server* s, double timeout_s, vfgpu_result* res) {
  if (!s || !res) return fail(VFGPU_ERR_INVALID, "vfgpu_server_next: null argument");
  std::unique_lock<std::mutex> lk(s->m);
  auto ready = [&] { return !s->done.empty(); };
  if (timeout_s < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
    return VFGPU_NOT_CONVERGED;
  *res = s->done.front();
  s->done.pop_front();
  return VFGPU_OK;
}

double vfgpu_server_clock(vfgpu_server* s) { return s ? s->now() : 0.0; }

int vfgpu_server_info_get(vfgpu_server* s, vfgpu_server_info* info) {
  if (!s || !info) return fail(VFGPU_ERR_INVALID, "vfgpu_server_info_get: null argument");
  std::lock_guard<std::mutex> lk(s->m);
  info->budget_bytes = s->budget;
  info->reserved_bytes = s->reserved;
  info->peak_reserved_bytes = s->peak_reserved;
  info->workers = s->nworkers;
  info->contexts = (int)s->pool.size();
  info->contexts_created = s->contexts_created;
  info->evictions = s->evictions;
  info->submitted = s->submitted;
  info->completed = s->completed;
  info->queued = (long long)s->queue.size();
  info->running = s->running;
  return VFGPU_OK;
}

int vfgpu_server_destroy(vfgpu_server* s) {
  if (!s) return VFGPU_OK;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv_job.notify_all();
  for (auto& t : s->workers) t.join();
  cudaSetDevice(s->dev);
  for (auto& sl : s->pool) vfgpu_destroy(sl.ctx);
  delete s;
  return VFGPU_OK;
}

}  // extern "C"
