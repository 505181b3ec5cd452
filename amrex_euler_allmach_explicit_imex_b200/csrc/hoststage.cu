// Copies between a caller's pageable host box and the device through the
// context's own page-locked staging buffers.
//
// A copy from pageable memory makes the CUDA driver stage it through a small
// pinned buffer of its own, one chunk at a time, behind the calling thread:
// at 2560x640 a state (52 MB) crosses at about 13 GB/s.  Here the rows of a
// band are first copied by a few host threads into a pinned staging copy of
// the state (compact: 4 planes of nx x ny), and the band then crosses by DMA
// while the threads copy the next band, so the host copies and the transfer
// overlap.  The staging buffers (one per direction) are allocated on the
// first pageable call and kept by the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"

// A fixed set of host threads that run the n tasks of one job together with
// the calling thread; run() returns when every task is done and no thread
// holds the job any more (the job lives on run()'s stack).
class CopyPool {
 public:
  explicit CopyPool(int workers)
  {
    for (int w = 0; w < workers; ++w) threads_.emplace_back([this] { loop(); });
  }
  ~CopyPool()
  {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  void run(int n, const std::function<void(int)>& f)
  {
    Job job;
    job.f = &f;
    job.n = n;
    {
      std::lock_guard<std::mutex> lock(mu_);
      job_ = &job;
      ++gen_;
    }
    cv_.notify_all();
    const int mine = drain(job);
    std::unique_lock<std::mutex> lock(mu_);
    job.done += mine;
    job_ = nullptr;  // no thread takes it from here on
    done_cv_.wait(lock, [&] { return job.done == job.n && job.users == 0; });
  }

 private:
  struct Job {
    const std::function<void(int)>* f = nullptr;
    int n = 0;
    std::atomic<int> next{0};
    int done = 0;   // tasks finished (under mu_)
    int users = 0;  // worker threads holding the job (under mu_)
  };
  static int drain(Job& j)
  {
    int k, count = 0;
    while ((k = j.next.fetch_add(1)) < j.n) {
      (*j.f)(k);
      ++count;
    }
    return count;
  }
  void loop()
  {
    unsigned long long seen = 0;
    for (;;) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        j = job_;
        if (!j) continue;
        ++j->users;
      }
      const int count = drain(*j);
      std::lock_guard<std::mutex> lock(mu_);
      j->done += count;
      --j->users;
      if (j->done == j->n && j->users == 0) done_cv_.notify_all();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  Job* job_ = nullptr;
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

struct HostStage {
  double* in = nullptr;   // pinned: what crosses to the device
  double* out = nullptr;  // pinned: what comes back
  size_t doubles = 0;
  CopyPool* pool = nullptr;
  ~HostStage()
  {
    delete pool;
    if (in) cudaFreeHost(in);
    if (out) cudaFreeHost(out);
  }
};

bool host_pageable(const void* p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // an unknown pointer is plain host memory
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

HostStage* host_stage(ecg_ctx* c)
{
  const size_t need = 4 * static_cast<size_t>(c->grid.nx) * static_cast<size_t>(c->grid.ny);
  if (c->stage && c->stage->doubles >= need) return c->stage;
  delete c->stage;
  c->stage = nullptr;
  HostStage* s = new HostStage();
  s->doubles = need;
  if (cudaMallocHost(&s->in, sizeof(double) * need) != cudaSuccess ||
      cudaMallocHost(&s->out, sizeof(double) * need) != cudaSuccess) {
    c->err = "pinned staging buffers: allocation failed";
    cudaGetLastError();
    delete s;
    return nullptr;
  }
  // three quarters of the host threads, with the caller (measured on a 16-thread
  // host at 2560x640: 3, 7, 11, 15 workers gave 0.40, 0.51, 0.62, 0.57 G
  // cell-updates/s through the host step)
  const unsigned hw = std::thread::hardware_concurrency();
  const int workers = std::max(1, std::min(15, static_cast<int>(hw * 3 / 4) - 1));
  s->pool = new CopyPool(workers);
  c->stage = s;
  return s;
}

void host_stage_destroy(HostStage* s) { delete s; }
double* host_stage_in(HostStage* s) { return s->in; }
double* host_stage_out(HostStage* s) { return s->out; }

// Rows [r0, r1) of the 4 planes: the caller's box (rows jstride apart, planes
// nstride apart, from its Array4 base already offset to cell (0, 0)) to the
// compact stage (to_stage), or back.  One task per plane and slice of rows.
void host_stage_copy(HostStage* s, double* stage, double* host, int64_t jstride, int64_t nstride, int nx, int ny,
                     int r0, int r1, bool to_stage)
{
  constexpr int kRowsPerTask = 16;
  const int rows = r1 - r0;
  if (rows <= 0) return;
  const int slices = (rows + kRowsPerTask - 1) / kRowsPerTask;
  const size_t plane = static_cast<size_t>(nx) * static_cast<size_t>(ny);
  const std::function<void(int)> job = [&](int k) {
    const int n = k / slices, sl = k % slices;
    const int a = r0 + sl * kRowsPerTask, b = std::min(r1, a + kRowsPerTask);
    for (int r = a; r < b; ++r) {
      double* st = stage + n * plane + static_cast<size_t>(r) * nx;
      double* h = host + n * nstride + static_cast<int64_t>(r) * jstride;
      if (to_stage) std::memcpy(st, h, sizeof(double) * nx);
      else std::memcpy(h, st, sizeof(double) * nx);
    }
  };
  s->pool->run(4 * slices, job);
}
