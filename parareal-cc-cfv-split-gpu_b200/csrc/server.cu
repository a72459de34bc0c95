// server.cu -- continuous-batching request loop over the multi-problem engine.
//
// A worker thread owns one MultiEngine on its own stream.  Each epoch it
//  1. admits queued requests in arrival order while their resident state fits
//     the HBM budget and a slot is free (a request larger than the whole
//     budget is rejected at submission with CCFV_ERR_BUDGET),
//  2. advances every resident problem by one Parareal iteration in shared
//     launches (newly admitted problems first run their coarse sweep),
//  3. retires the problems that converged: copies their result to the
//     caller's buffer, releases their device memory and wakes waiters.
// Requests that arrive while others are running join at the next epoch, so
// their work overlaps on the device with the work already resident.
#include <chrono>
#include <cstdint>
#include <new>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "multi.h"

using Clock = std::chrono::steady_clock;

namespace {

struct Request {
  uint64_t ticket = 0;
  ccfv_problem p;
  size_t bytes = 0;
  int state = CCFV_REQ_QUEUED;
  int rc = CCFV_OK;
  int slot = -1;
  bool cancel = false;
  ccfv_stats stats;
  Clock::time_point t_submit, t_done;
};

}  // namespace

struct ccfv_server {
  ccfv_server_opts opts;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  size_t used = 0;
  int active = 0;
  bool stop = false;
  uint64_t next = 1;
  int fatal = CCFV_OK;
};

namespace {

void serve(ccfv_server *S) {
  using namespace ccfv;
  cudaSetDevice(S->opts.device);
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->fatal = CCFV_ERR_CUDA;
    S->cv_done.notify_all();
    return;
  }
  {
    MultiEngine E(S->opts.device, st);
    std::unordered_map<int, Request *> by_slot;
    std::vector<int> fin;
    for (;;) {
      std::vector<Request *> admit;
      {
        std::unique_lock<std::mutex> lk(S->mu);
        // drop cancelled requests that are still queued
        for (auto it = S->queue.begin(); it != S->queue.end();) {
          if ((*it)->cancel) {
            (*it)->state = CCFV_REQ_CANCELLED;
            (*it)->rc = CCFV_ERR_CANCELLED;
            (*it)->t_done = Clock::now();
            it = S->queue.erase(it);
            S->cv_done.notify_all();
          } else {
            ++it;
          }
        }
        while (!S->queue.empty()) {
          Request *r = S->queue.front();
          if (S->used + r->bytes > S->opts.hbm_budget_bytes) break;
          if (S->opts.max_active > 0 && S->active >= S->opts.max_active) break;
          S->queue.pop_front();
          S->used += r->bytes;
          S->active += 1;
          r->state = CCFV_REQ_RUNNING;
          admit.push_back(r);
        }
        if (admit.empty() && by_slot.empty()) {
          if (S->stop) break;
          S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
          continue;
        }
      }
      for (Request *r : admit) {
        int slot = -1;
        int rc = E.add(r->p, &slot);
        if (rc) {
          std::lock_guard<std::mutex> lk(S->mu);
          r->rc = rc;
          r->state = CCFV_REQ_FAILED;
          r->t_done = Clock::now();
          S->used -= r->bytes;
          S->active -= 1;
          S->cv_done.notify_all();
          continue;
        }
        r->slot = slot;
        by_slot[slot] = r;
      }
      if (by_slot.empty()) continue;
      int rc = E.iterate(&fin);
      if (rc) {  // device-level failure: fail every resident request
        std::lock_guard<std::mutex> lk(S->mu);
        for (auto &kv : by_slot) {
          kv.second->rc = rc;
          kv.second->state = CCFV_REQ_FAILED;
          kv.second->t_done = Clock::now();
          E.remove(kv.first);
          S->used -= kv.second->bytes;
          S->active -= 1;
        }
        by_slot.clear();
        S->cv_done.notify_all();
        continue;
      }
      // cancelled running requests leave at the epoch boundary
      std::vector<int> leave;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        for (auto &kv : by_slot)
          if (kv.second->cancel) leave.push_back(kv.first);
      }
      for (int sl : fin) E.finish(sl);
      cudaStreamSynchronize(st);
      std::lock_guard<std::mutex> lk(S->mu);
      const auto now = Clock::now();
      for (int sl : fin) {
        Request *r = by_slot[sl];
        ccfv::fill_stats(*E.get(sl), &r->stats,
                         std::chrono::duration<double, std::milli>(now - r->t_submit).count());
        r->state = CCFV_REQ_DONE;
        r->t_done = now;
        E.remove(sl);
        by_slot.erase(sl);
        S->used -= r->bytes;
        S->active -= 1;
      }
      for (int sl : leave) {
        auto it = by_slot.find(sl);
        if (it == by_slot.end()) continue;
        it->second->state = CCFV_REQ_CANCELLED;
        it->second->rc = CCFV_ERR_CANCELLED;
        it->second->t_done = now;
        E.remove(sl);
        S->used -= it->second->bytes;
        S->active -= 1;
        by_slot.erase(it);
      }
      S->cv_done.notify_all();
    }
  }
  cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

int ccfv_server_create(ccfv_server **out, const ccfv_server_opts *opts) {
  if (!out || !opts || opts->hbm_budget_bytes == 0) return CCFV_ERR_INVALID;
  ccfv_server *S = new (std::nothrow) ccfv_server();
  if (!S) return CCFV_ERR_NOMEM;
  S->opts = *opts;
  if (cudaSetDevice(opts->device) != cudaSuccess) {
    delete S;
    return CCFV_ERR_CUDA;
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, opts->device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;  // keep freed slice states cached in the pool
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  S->worker = std::thread(serve, S);
  *out = S;
  return CCFV_OK;
}

int ccfv_server_submit(ccfv_server *S, const ccfv_problem *p, uint64_t *ticket) {
  if (!S || !p || !ticket || !p->C0 || !p->C_T) return CCFV_ERR_INVALID;
  ccfv::Problem probe;
  std::string err;
  int rc = ccfv::problem_setup(probe, *p, &err);
  if (rc) return rc;
  auto r = std::make_unique<Request>();
  r->p = *p;
  r->bytes = probe.bytes;
  if (r->bytes > S->opts.hbm_budget_bytes) return CCFV_ERR_BUDGET;
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return S->fatal;
  r->ticket = S->next++;
  *ticket = r->ticket;
  S->queue.push_back(r.get());
  S->reqs[r->ticket] = std::move(r);
  S->cv_work.notify_one();
  return CCFV_OK;
}

static int report(Request *r, int *state, ccfv_stats *stats, double *latency_ms) {
  if (state) *state = r->state;
  if (r->state == CCFV_REQ_DONE || r->state == CCFV_REQ_FAILED || r->state == CCFV_REQ_CANCELLED) {
    if (stats) *stats = r->stats;
    if (latency_ms)
      *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  }
  return r->state == CCFV_REQ_FAILED || r->state == CCFV_REQ_CANCELLED ? r->rc : CCFV_OK;
}

int ccfv_server_poll(ccfv_server *S, uint64_t ticket, int *state, ccfv_stats *stats,
                     double *latency_ms) {
  if (!S) return CCFV_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return CCFV_ERR_NOT_FOUND;
  return report(it->second.get(), state, stats, latency_ms);
}

int ccfv_server_wait(ccfv_server *S, uint64_t ticket, double timeout_s, ccfv_stats *stats,
                     double *latency_ms) {
  if (!S) return CCFV_ERR_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return CCFV_ERR_NOT_FOUND;
  Request *r = it->second.get();
  auto finished = [&] {
    return S->fatal || r->state == CCFV_REQ_DONE || r->state == CCFV_REQ_FAILED ||
           r->state == CCFV_REQ_CANCELLED;
  };
  if (timeout_s > 0) {
    if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), finished))
      return CCFV_ERR_TIMEOUT;
  } else {
    S->cv_done.wait(lk, finished);
  }
  if (S->fatal && r->state != CCFV_REQ_DONE) return S->fatal;
  return report(r, nullptr, stats, latency_ms);
}

int ccfv_server_cancel(ccfv_server *S, uint64_t ticket) {
  if (!S) return CCFV_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return CCFV_ERR_NOT_FOUND;
  it->second->cancel = true;
  S->cv_work.notify_one();
  return CCFV_OK;
}

int ccfv_server_info(ccfv_server *S, size_t *used_bytes, int *active, int *queued) {
  if (!S) return CCFV_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  if (used_bytes) *used_bytes = S->used;
  if (active) *active = S->active;
  if (queued) *queued = (int)S->queue.size();
  return CCFV_OK;
}

int ccfv_server_destroy(ccfv_server *S) {
  if (!S) return CCFV_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    for (Request *r : S->queue) r->cancel = true;
    S->cv_work.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  delete S;
  return CCFV_OK;
}

}  // extern "C"
