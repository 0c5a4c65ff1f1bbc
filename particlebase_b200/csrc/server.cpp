// Serving loop (pb_srv_*, include/pb/pb.h): a scheduler thread that keeps one
// batch of MD jobs resident on the device and packs new jobs into it as they
// arrive and memory frees up.
//
// Chunk boundary protocol (all in the scheduler thread):
//   1. jobs whose step budget ran out during the last chunk are copied to host
//      memory and leave the batch;
//   2. queued jobs are admitted in FIFO order while the memory estimate of the
//      resident set (old and new batch both, since a repack holds both for a
//      moment) stays within the budget and the atom / job caps;
//   3. if the membership changed, the batch is repacked: continuing jobs keep
//      their device state bit for bit, new jobs are imported, cells are set up
//      and every job's remaining step count becomes its step budget;
//   4. the batch advances by K whole steps (graph replays), K chosen so a
//      chunk takes about max(chunk_ms, 4 x the last repack time) of GPU time
//      but no longer than the longest remaining job needs.
// Jobs whose budget ends inside a chunk simply stop there (the kernels skip
// them), so every job runs exactly its own step count.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pb/pb.h"

namespace {

struct Job {
  uint64_t id = 0;
  int state = PB_JOB_QUEUED;
  uint32_t n = 0, steps = 0, ntypes = 1;
  float cell[6] = {0, 0, 0, 0, 0, 0};
  float rc = 0, dt = 0, kB = 1;
  std::vector<float> lj, ljcut;
  std::vector<double> r3, v3, mass;
  std::vector<uint32_t> type;
  size_t bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  uint32_t status = 0;
  uint32_t remaining = 0;  // steps still to run while resident
  // result
  std::vector<float> r4, F4;
  std::vector<unsigned char> v;
};

}  // namespace

struct pb_srv {
  pb_srv_config cfg{};
  int device = 0;
  size_t budget = 0;
  std::chrono::steady_clock::time_point t0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::string err;
  uint64_t next_id = 1;
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Job>> jobs;
  std::vector<uint64_t> finished_unpolled;
  uint64_t outstanding = 0;  // queued + running
  pb_srv_stats st{};

  // scheduler-thread state
  pb_batch *batch = nullptr;
  std::vector<Job *> slots;  // job of each batch system
  double ms_per_atom_step = 5e-7;
  double last_repack_ms = 0.0;
  bool trace = false;  // PB_SRV_TRACE: per-repack phase times on stderr
  bool reserved = false;  // the pool took reserve_bytes at creation
  std::thread worker;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

size_t job_bytes(const pb_srv_job &j, uint32_t flags) {
  size_t b = 0;
  const float rmax = j.rc;
  if (pb_batch_estimate_bytes(&j.natoms, j.cell6, &rmax, 1, flags, &b) != PB_OK) return 0;
  return b + 4 * (size_t)j.natoms;  // system id per atom once batched
}

// Copy a finished job's state out of the batch (scheduler thread, lock not held).
int collect(pb_srv *s, uint32_t slot, Job &j) {
  const uint32_t n = j.n;
  j.r4.resize(4 * (size_t)n);
  j.F4.resize(4 * (size_t)n);
  int rc = pb_batch_get(s->batch, slot, PB_FIELD_R, j.r4.data(), 16 * (size_t)n);
  if (!rc) rc = pb_batch_get(s->batch, slot, PB_FIELD_F, j.F4.data(), 16 * (size_t)n);
  if (!rc) {
    if (s->cfg.flags & PB_MD_VEL_FP64) {
      j.v.resize(24 * (size_t)n);
      rc = pb_batch_get(s->batch, slot, PB_FIELD_VD, j.v.data(), j.v.size());
    } else {
      j.v.resize(16 * (size_t)n);
      rc = pb_batch_get(s->batch, slot, PB_FIELD_V, j.v.data(), j.v.size());
    }
  }
  return rc;
}

int setup_new(pb_batch *b, uint32_t k, const Job &j) {
  int rc = pb_batch_set_system(b, k, j.cell, j.rc, j.lj.data(), j.ntypes, j.dt, j.kB);
  if (!rc && !j.ljcut.empty()) rc = pb_batch_set_lj_cut(b, k, j.ljcut.data(), j.ntypes);
  if (!rc)
    rc = pb_batch_import(b, k, j.r3.data(), j.v3.empty() ? nullptr : j.v3.data(),
                         j.mass.empty() ? nullptr : j.mass.data(),
                         j.type.empty() ? nullptr : j.type.data());
  return rc;
}

void fail_resident(pb_srv *s, const std::string &why) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->err = why;
  for (Job *j : s->slots) {
    j->state = PB_JOB_FAILED;
    j->t_done = s->now();
    s->finished_unpolled.push_back(j->id);
    ++s->st.failed;
    --s->outstanding;
  }
  s->slots.clear();
  if (s->batch) pb_batch_destroy(s->batch);
  s->batch = nullptr;
  s->cv_done.notify_all();
}

void scheduler(pb_srv *s) {
  cudaSetDevice(s->device);
  for (;;) {
    // ---- 1. retire finished jobs
    std::vector<uint32_t> keep;
    std::vector<Job *> done;
    for (uint32_t k = 0; k < s->slots.size(); ++k) {
      if (s->slots[k]->remaining == 0)
        done.push_back(s->slots[k]);
      else
        keep.push_back(k);
    }
    bool failed = false;
    for (uint32_t k = 0; k < s->slots.size() && !failed; ++k)
      if (s->slots[k]->remaining == 0 && collect(s, k, *s->slots[k]) != PB_OK) failed = true;
    if (failed) {
      fail_resident(s, std::string("collect: ") + pb_batch_last_error(s->batch));
      continue;
    }

    // ---- 2. admit
    std::vector<Job *> admit;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (Job *j : done) {
        j->state = PB_JOB_DONE;
        j->t_done = s->now();
        s->finished_unpolled.push_back(j->id);
        ++s->st.done;
        s->st.atom_steps += (double)j->n * j->steps;
        --s->outstanding;
      }
      if (!done.empty()) s->cv_done.notify_all();
      if (keep.empty() && s->queue.empty()) {
        if (s->batch) {
          pb_batch_destroy(s->batch);
          s->batch = nullptr;
          s->slots.clear();
        }
        s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      }
      if (s->stop) break;
      size_t old_bytes = 0, new_bytes = 0;
      uint64_t atoms = 0;
      for (Job *j : s->slots) old_bytes += j->bytes;
      for (uint32_t k : keep) {
        new_bytes += s->slots[k]->bytes;
        atoms += s->slots[k]->n;
      }
      uint32_t njobs = (uint32_t)keep.size();
      while (!s->queue.empty()) {
        Job *j = s->jobs[s->queue.front()].get();
        const bool fits = old_bytes + new_bytes + j->bytes <= s->budget &&
                          (!s->cfg.max_atoms || atoms + j->n <= s->cfg.max_atoms || njobs == 0) &&
                          (!s->cfg.max_jobs || njobs + 1 <= s->cfg.max_jobs);
        if (!fits) break;
        s->queue.pop_front();
        admit.push_back(j);
        new_bytes += j->bytes;
        atoms += j->n;
        ++njobs;
      }
      s->st.peak_bytes = std::max(s->st.peak_bytes, new_bytes);
      s->st.peak_jobs = std::max<uint64_t>(s->st.peak_jobs, njobs);
      s->st.peak_atoms = std::max<uint64_t>(s->st.peak_atoms, atoms);
    }

    // ---- 3. repack when membership changed
    if ((!done.empty() || !admit.empty()) && keep.empty() && admit.empty()) {
      pb_batch_destroy(s->batch);  // everything finished and nothing fits yet
      s->batch = nullptr;
      std::lock_guard<std::mutex> lk(s->mu);
      s->slots.clear();
      continue;
    }
    if (!done.empty() || !admit.empty()) {
      const auto t_r = std::chrono::steady_clock::now();
      const uint32_t nsys = (uint32_t)(keep.size() + admit.size());
      std::vector<int32_t> src(nsys, -1);
      std::vector<uint32_t> nat(nsys, 0);
      std::vector<Job *> slots(nsys);
      for (uint32_t k = 0; k < keep.size(); ++k) {
        src[k] = (int32_t)keep[k];
        slots[k] = s->slots[keep[k]];
      }
      for (uint32_t a = 0; a < admit.size(); ++a) {
        const uint32_t k = (uint32_t)keep.size() + a;
        nat[k] = admit[a]->n;
        slots[k] = admit[a];
      }
      pb_batch *nb = nullptr;
      int rc;
      auto lap = [t = std::chrono::steady_clock::now()]() mutable {
        const auto n = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(n - t).count();
        t = n;
        return ms;
      };
      double ph[5] = {0, 0, 0, 0, 0};
      if (s->batch && !keep.empty()) {
        rc = pb_batch_repack(s->batch, src.data(), nat.data(), nsys, &nb);
      } else {
        rc = pb_batch_create(nat.data(), nsys, s->cfg.flags, &nb);
        if (!rc)
          rc = pb_batch_set_tuning(nb, s->cfg.force_threads ? s->cfg.force_threads : 256,
                                   s->cfg.seg_scale > 0 ? s->cfg.seg_scale : 1.0f);
      }
      std::string why = rc ? std::string("repack: ") + (s->batch ? pb_batch_last_error(s->batch) : "")
                           : std::string();
      ph[0] = lap();
      for (uint32_t a = 0; a < admit.size() && !rc; ++a) {
        rc = setup_new(nb, (uint32_t)keep.size() + a, *admit[a]);
        if (rc) why = std::string("admit: ") + pb_batch_last_error(nb);
      }
      ph[1] = lap();
      if (!rc) {
        rc = pb_batch_setup_cells(nb, nullptr);
        if (rc) why = std::string("setup_cells: ") + pb_batch_last_error(nb);
      }
      ph[2] = lap();
      std::vector<uint32_t> rem(nsys);
      for (uint32_t k = 0; k < nsys; ++k) rem[k] = slots[k]->remaining;
      if (!rc) rc = pb_batch_set_steps_left(nb, rem.data());
      ph[3] = lap();
      if (s->batch) pb_batch_destroy(s->batch);
      s->batch = nb;
      ph[4] = lap();
      if (s->trace) {
        uint64_t natoms = 0;
        for (Job *j : slots) natoms += j->n;
        std::fprintf(stderr,
                     "pb_srv repack: %u jobs (%zu kept, %zu new, %zu done), %llu atoms; ms: "
                     "repack %.2f admit %.2f cells %.2f budgets %.2f free %.2f\n",
                     nsys, keep.size(), admit.size(), done.size(), (unsigned long long)natoms,
                     ph[0], ph[1], ph[2], ph[3], ph[4]);
      }
      {
        std::lock_guard<std::mutex> lk(s->mu);
        s->slots = slots;
        const double t = s->now();
        for (Job *j : admit) {
          j->state = PB_JOB_RUNNING;
          j->t_admit = t;
        }
        ++s->st.repacks;
        const double sec =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t_r).count();
        s->st.repack_seconds += sec;
        s->last_repack_ms = 1e3 * sec;
      }
      if (rc) {
        fail_resident(s, why);
        continue;
      }
    }
    if (s->slots.empty()) continue;

    // ---- 4. one chunk of whole steps
    uint64_t atoms = 0;
    uint32_t longest = 0;
    for (Job *j : s->slots) {
      atoms += j->n;
      longest = std::max(longest, j->remaining);
    }
    // a chunk lasts at least four repacks, so repacking costs at most a fifth
    // of the GPU time even when jobs arrive and leave at every boundary
    const double chunk_ms =
        std::max(s->cfg.chunk_ms > 0 ? (double)s->cfg.chunk_ms : 100.0, 4.0 * s->last_repack_ms);
    double want = chunk_ms / std::max(1e-6, s->ms_per_atom_step * (double)atoms);
    uint32_t K = (uint32_t)std::max(2.0, std::min(want, 1e6));
    K += K & 1u;
    K = std::min(K, longest);
    float ms = 0.f;
    int rc = pb_batch_run_timed(s->batch, s->cfg.mode, K, &ms);
    if (rc) {
      fail_resident(s, std::string("run: ") + pb_batch_last_error(s->batch));
      continue;
    }
    std::vector<uint32_t> bits(s->slots.size());
    pb_batch_status(s->batch, bits.data());
    s->ms_per_atom_step = std::max(1e-9, (double)ms / ((double)K * (double)atoms));
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->st.gpu_seconds += ms / 1e3;
      ++s->st.chunks;
      for (uint32_t k = 0; k < s->slots.size(); ++k) {
        Job *j = s->slots[k];
        j->status |= bits[k];
        j->remaining -= std::min(j->remaining, K);
      }
    }
  }
}

}  // namespace

extern "C" {

int pb_srv_create(const pb_srv_config *cfg, pb_srv **out) {
  if (!cfg || !out) return PB_ERR_ARG;
  if (cfg->mode != PB_MODE_VV && cfg->mode != PB_MODE_GAUSS) return PB_ERR_ARG;
  if (cfg->mode == PB_MODE_VV && (cfg->flags & PB_MD_VEL_FP64)) return PB_ERR_UNSUPPORTED;
  *out = nullptr;
  auto *s = new pb_srv;
  s->cfg = *cfg;
  s->t0 = std::chrono::steady_clock::now();
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return PB_ERR_CUDA;
  }
  s->budget = cfg->hbm_budget;
  if (!s->budget) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      delete s;
      return PB_ERR_CUDA;
    }
    s->budget = (size_t)(0.9 * (double)fr);
  }
  if (const char *t = std::getenv("PB_SRV_TRACE")) s->trace = t[0] && t[0] != '0';
  if (cfg->reserve_bytes)  // without the memory free, the server grows the pool as it goes
    s->reserved = pb_pool_reserve(std::min(cfg->reserve_bytes, s->budget)) == PB_OK;
  s->worker = std::thread(scheduler, s);
  *out = s;
  return PB_OK;
}

int pb_srv_destroy(pb_srv *s) {
  if (!s) return PB_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->batch) pb_batch_destroy(s->batch);
  if (s->reserved) pb_pool_trim();
  delete s;
  return PB_OK;
}

int pb_srv_submit(pb_srv *s, const pb_srv_job *job, uint64_t *id) {
  if (!s || !job || !job->r3 || !job->sigma_eps || job->natoms == 0 || job->ntypes == 0)
    return PB_ERR_ARG;
  auto j = std::make_unique<Job>();
  const uint32_t n = job->natoms, nt = job->ntypes;
  j->n = n;
  j->steps = job->steps;
  j->remaining = job->steps;
  j->ntypes = nt;
  std::memcpy(j->cell, job->cell6, sizeof(j->cell));
  j->rc = job->rc;
  j->dt = job->dt;
  j->kB = job->kB > 0 ? job->kB : 1.0f;
  j->lj.assign(job->sigma_eps, job->sigma_eps + 2 * nt * nt);
  if (job->sigma_eps_rc) j->ljcut.assign(job->sigma_eps_rc, job->sigma_eps_rc + 3 * nt * nt);
  j->r3.assign(job->r3, job->r3 + 3 * (size_t)n);
  if (job->v3) j->v3.assign(job->v3, job->v3 + 3 * (size_t)n);
  if (job->mass) j->mass.assign(job->mass, job->mass + n);
  if (job->type) j->type.assign(job->type, job->type + n);
  j->bytes = job_bytes(*job, s->cfg.flags);
  std::lock_guard<std::mutex> lk(s->mu);
  if (j->bytes == 0) {
    s->err = "job grid invalid (fewer than 3 cells per axis?)";
    ++s->st.rejected;
    return PB_ERR_ARG;
  }
  if (2 * j->bytes > s->budget) {  // a repack holds a job twice for a moment
    s->err = "job larger than the memory budget";
    ++s->st.rejected;
    return PB_ERR_OOM;
  }
  j->id = s->next_id++;
  j->t_submit = s->now();
  if (id) *id = j->id;
  ++s->st.submitted;
  ++s->outstanding;
  if (j->steps == 0) {  // nothing to run: the result is the input
    j->state = PB_JOB_DONE;
    j->t_admit = j->t_done = j->t_submit;
    j->r4.assign(4 * (size_t)n, 0.f);
    for (uint32_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) j->r4[4 * i + k] = (float)j->r3[3 * i + k];
    --s->outstanding;
    ++s->st.done;
    s->finished_unpolled.push_back(j->id);
    s->jobs[j->id] = std::move(j);
    s->cv_done.notify_all();
    return PB_OK;
  }
  s->queue.push_back(j->id);
  s->jobs[j->id] = std::move(j);
  s->cv_work.notify_all();
  return PB_OK;
}

int pb_srv_wait(pb_srv *s, uint64_t id, double timeout_s) {
  if (!s) return PB_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return PB_ERR_NOTFOUND;
  Job *j = it->second.get();
  auto ready = [&] { return j->state == PB_JOB_DONE || j->state == PB_JOB_FAILED; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
    return PB_ERR_STATE;
  return j->state == PB_JOB_DONE ? PB_OK : PB_ERR_DEVICE;
}

int pb_srv_drain(pb_srv *s, double timeout_s) {
  if (!s) return PB_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] { return s->outstanding == 0; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
    return PB_ERR_STATE;
  return PB_OK;
}

int pb_srv_poll(pb_srv *s, uint64_t *ids, uint32_t max, uint32_t *n) {
  if (!s || !n || (max && !ids)) return PB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  const uint32_t k = (uint32_t)std::min<size_t>(max, s->finished_unpolled.size());
  for (uint32_t i = 0; i < k; ++i) ids[i] = s->finished_unpolled[i];
  s->finished_unpolled.erase(s->finished_unpolled.begin(), s->finished_unpolled.begin() + k);
  *n = k;
  return PB_OK;
}

int pb_srv_info(pb_srv *s, uint64_t id, pb_srv_job_info *info) {
  if (!s || !info) return PB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return PB_ERR_NOTFOUND;
  const Job &j = *it->second;
  info->id = j.id;
  info->state = j.state;
  info->natoms = j.n;
  info->steps = j.steps;
  info->t_submit = j.t_submit;
  info->t_admit = j.t_admit;
  info->t_done = j.t_done;
  info->device_status = j.status;
  return PB_OK;
}

int pb_srv_result(pb_srv *s, uint64_t id, void *r4, void *v, size_t vbytes, void *F4) {
  if (!s) return PB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return PB_ERR_NOTFOUND;
  const Job &j = *it->second;
  if (j.state != PB_JOB_DONE) return PB_ERR_STATE;
  if (r4) std::memcpy(r4, j.r4.data(), 16 * (size_t)j.n);
  if (F4) {
    if (j.F4.empty()) return PB_ERR_STATE;
    std::memcpy(F4, j.F4.data(), 16 * (size_t)j.n);
  }
  if (v) {
    if (j.v.size() != vbytes) return PB_ERR_ARG;
    std::memcpy(v, j.v.data(), vbytes);
  }
  return PB_OK;
}

int pb_srv_release(pb_srv *s, uint64_t id) {
  if (!s) return PB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return PB_ERR_NOTFOUND;
  if (it->second->state != PB_JOB_DONE && it->second->state != PB_JOB_FAILED) return PB_ERR_STATE;
  s->jobs.erase(it);
  return PB_OK;
}

int pb_srv_stats_get(pb_srv *s, pb_srv_stats *st) {
  if (!s || !st) return PB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->st;
  return PB_OK;
}

double pb_srv_now(const pb_srv *s) { return s ? s->now() : 0.0; }

const char *pb_srv_last_error(const pb_srv *s) { return s ? s->err.c_str() : "null handle"; }

}  // extern "C"
