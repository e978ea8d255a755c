// lv_server.cuh -- the serving loop (lv_server_* in include/louvain_b200.h). Included at the end
// of lv_engine.cu, after lv::Run.
//
// Continuous batching with graph state resident in HBM: `max_slots` worker threads, each with
// its own CUDA stream, take requests from a FIFO queue as soon as a slot is free and the
// requests' device footprint fits the memory budget next to the requests already running.
// A slot takes the head of the queue together with the other queued small requests and runs
// them as one packed batch (every graph of a batch gets exactly the result it gets alone);
// batches on different slots overlap on the device, and device memory comes from the
// context's pool, so steady-state serving allocates nothing. Results stay on the host until
// polled. The reference has no counterpart (it runs one graph per call).
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace lv {

struct Request {
  int64_t id = 0;
  int64_t n = 0, E = 0;
  std::vector<int64_t> row;
  std::vector<int32_t> col;
  std::vector<float> w;
  // borrowed requests: the caller's buffers, valid until the request is polled done
  const int64_t* brow = nullptr;
  const int32_t* bcol = nullptr;
  const float* bw = nullptr;
  bool weighted = false;
  std::vector<int32_t> out;
  double modularity = 0;
  int32_t n_comm = 0;
  int state = 0;  // 0 queued, 1 running, 2 done
  lv_status status = LV_OK;
  std::string err;
  size_t est_bytes = 0;
  std::chrono::steady_clock::time_point t_submit, t_done;
};

// Device bytes a run of this size holds: 16 B per CSR entry (two entry buffers of destination
// and weight) and about 124 B per vertex of state and scratch, plus the control block.
inline size_t footprint(int64_t n, int64_t E) {
  return (size_t)E * 16 + (size_t)n * 124 + (size_t)(1u << 20) + sizeof(Ctrl);
}

}  // namespace lv

struct lv_server {
  lv_context* ctx = nullptr;
  int64_t budget = 0;
  int max_slots = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<lv::Request*> queue;
  std::unordered_map<int64_t, std::unique_ptr<lv::Request>> all;
  int64_t next_id = 1, n_done = 0, n_running = 0;
  int64_t used_bytes = 0;
  bool stop = false;
  std::vector<std::thread> workers;
  std::vector<cudaStream_t> streams;
  std::vector<uint32_t*> pinned;  // per slot: 64-byte readback buffer
  std::vector<std::unique_ptr<lv::DevSlot>> dslots;  // per slot: Dev buffer and captured graph

  // Continuous batching: a free slot takes the request at the head of the queue and, when
  // that request is small, every further queued request (in arrival order) that is small too,
  // of the same weight kind, fits the batch limits and fits the memory budget. The taken
  // requests run as one packed batch on the slot's stream; requests that arrive meanwhile wait
  // for the next free slot.
  static constexpr int64_t kSmallEntries = 1 << 22;   // requests up to 4M CSR entries batch
  static constexpr int64_t kBatchEntries = 1 << 24;   // at most 16M entries per batch
  static constexpr size_t kBatchGraphs = 1024;

  void worker(int slot) {
    cudaSetDevice(ctx->device);
    std::vector<lv::Request*> batch;
    for (;;) {
      batch.clear();
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return stop || (!queue.empty() && used_bytes + (int64_t)queue.front()->est_bytes <= budget);
        });
        if (stop && queue.empty()) return;
        if (queue.empty() || used_bytes + (int64_t)queue.front()->est_bytes > budget) continue;
        lv::Request* r0 = queue.front();
        queue.pop_front();
        batch.push_back(r0);
        used_bytes += (int64_t)r0->est_bytes;
        // a graph batches only while one edge chunk covers it (the chunk rule of a single run
        // then never splits its pass, so the batch result is the single-run result)
        const int64_t chunk = ctx->cfg.chunk_edges > 0 ? ctx->cfg.chunk_edges : kSmallEntries;
        const int64_t small = std::min<int64_t>(kSmallEntries, chunk);
        if (r0->E <= small) {
          int64_t entries = r0->E;
          for (auto it = queue.begin(); it != queue.end() && batch.size() < kBatchGraphs;) {
            lv::Request* r = *it;
            if (r->E <= small && r->weighted == r0->weighted &&
                entries + r->E <= kBatchEntries && used_bytes + (int64_t)r->est_bytes <= budget) {
              batch.push_back(r);
              entries += r->E;
              used_bytes += (int64_t)r->est_bytes;
              it = queue.erase(it);
            } else {
              ++it;
            }
          }
        }
        for (lv::Request* r : batch) r->state = 1;
        n_running += (int64_t)batch.size();
      }
      run_batch(batch, slot);
      {
        std::lock_guard<std::mutex> lk(mu);
        const auto now = std::chrono::steady_clock::now();
        for (lv::Request* r : batch) {
          used_bytes -= (int64_t)r->est_bytes;
          r->state = 2;
          r->t_done = now;
          // the request's input is no longer needed
          std::vector<int64_t>().swap(r->row);
          std::vector<int32_t>().swap(r->col);
          std::vector<float>().swap(r->w);
          r->brow = nullptr;
          r->bcol = nullptr;
          r->bw = nullptr;
        }
        n_running -= (int64_t)batch.size();
        n_done += (int64_t)batch.size();
      }
      cv_work.notify_all();
      cv_done.notify_all();
    }
  }

  void run_batch(const std::vector<lv::Request*>& batch, int slot) {
    try {
      lv::Run run(ctx, streams[slot], pinned[slot], dslots[slot].get());
      std::vector<lv::Run::Piece> ps;
      ps.reserve(batch.size());
      for (lv::Request* r : batch) {
        const bool b = r->brow != nullptr;
        ps.push_back({r->n, r->E, b ? r->brow : r->row.data(), b ? r->bcol : r->col.data(),
                      r->weighted ? (b ? r->bw : r->w.data()) : nullptr});
      }
      run.init_pieces(ps);
      run.louvain();
      std::vector<lv::GraphState> gs(batch.size());
      int64_t vb = 0;
      for (lv::Request* r : batch) {
        r->out.resize((size_t)r->n);
        LV_CUDA(cudaMemcpyAsync(r->out.data(), run.D.out + vb, (size_t)r->n * 4, cudaMemcpyDeviceToHost, run.st));
        vb += r->n;
      }
      LV_CUDA(cudaMemcpyAsync(gs.data(), run.D.gs, sizeof(lv::GraphState) * batch.size(),
                              cudaMemcpyDeviceToHost, run.st));
      LV_CUDA(cudaStreamSynchronize(run.st));
      for (size_t i = 0; i < batch.size(); ++i) {
        batch[i]->modularity = gs[i].Q;
        batch[i]->n_comm = (int32_t)gs[i].n_best;
        batch[i]->status = LV_OK;
      }
    } catch (const lv::Fail& f) {
      for (lv::Request* r : batch) {
        r->status = f.st;
        r->err = f.msg;
      }
      cudaGetLastError();
    } catch (const std::bad_alloc&) {
      for (lv::Request* r : batch) {
        r->status = LV_ERR_NOMEM;
        r->err = "host allocation failed";
      }
    }
  }
};

extern "C" {

lv_status lv_server_create(lv_context* ctx, int64_t budget_bytes, int32_t max_slots, lv_server** out) {
  if (!ctx || !out || budget_bytes <= 0 || max_slots <= 0 || max_slots > 64) return LV_ERR_ARGUMENT;
  *out = nullptr;
  // the serving slots run concurrently and the refine view has one device slot per context
  if (ctx->cfg.refine) {
    ctx->err = "the server does not run refining configurations";
    return LV_ERR_ARGUMENT;
  }
  auto s = std::make_unique<lv_server>();
  s->ctx = ctx;
  s->budget = budget_bytes;
  s->max_slots = max_slots;
  cudaSetDevice(ctx->device);
  for (int i = 0; i < max_slots; ++i) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
      cudaGetLastError();
      return LV_ERR_CUDA;
    }
    s->streams.push_back(st);
    uint32_t* pb = nullptr;
    if (cudaMallocHost(&pb, 64) != cudaSuccess) {
      for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
      for (uint32_t* x : s->pinned) cudaFreeHost(x);
      cudaGetLastError();
      return LV_ERR_CUDA;
    }
    s->pinned.push_back(pb);
    auto ds = std::make_unique<lv::DevSlot>();
    if (ds->create() != cudaSuccess) {
      for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
      for (uint32_t* x : s->pinned) cudaFreeHost(x);
      for (auto& d : s->dslots) d->destroy();
      cudaGetLastError();
      return LV_ERR_CUDA;
    }
    s->dslots.push_back(std::move(ds));
  }
  lv_server* p = s.get();
  for (int i = 0; i < max_slots; ++i) s->workers.emplace_back([p, i] { p->worker(i); });
  *out = s.release();
  return LV_OK;
}

lv_status lv_server_destroy(lv_server* s) {
  if (!s) return LV_ERR_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    // queued requests that never started are dropped
    for (lv::Request* r : s->queue) {
      r->state = 2;
      r->status = LV_ERR_STATE;
      r->err = "server destroyed before the request started";
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
  for (uint32_t* pb : s->pinned) cudaFreeHost(pb);
  for (auto& d : s->dslots) d->destroy();
  delete s;
  return LV_OK;
}

static lv_status server_submit(lv_server* s, int64_t n, const int64_t* row_ptr, const int32_t* col,
                               const float* w, bool borrow, int64_t* request_id) {
  if (!s || !row_ptr || !col || !request_id || n <= 0) return LV_ERR_ARGUMENT;
  const int64_t E = row_ptr[n];
  if (row_ptr[0] != 0) return LV_ERR_INPUT;
  if (E <= 0 || E > (1ll << 30)) return LV_ERR_RANGE;
  auto r = std::make_unique<lv::Request>();
  r->n = n;
  r->E = E;
  r->est_bytes = lv::footprint(n, E);
  if ((int64_t)r->est_bytes > s->budget) return LV_ERR_BUDGET;
  r->t_submit = std::chrono::steady_clock::now();
  r->weighted = w != nullptr;
  if (borrow) {
    r->brow = row_ptr;
    r->bcol = col;
    r->bw = w;
  } else {
    r->row.assign(row_ptr, row_ptr + n + 1);
    r->col.assign(col, col + E);
    if (w) r->w.assign(w, w + E);
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return LV_ERR_STATE;
    r->id = s->next_id++;
    *request_id = r->id;
    s->queue.push_back(r.get());
    s->all.emplace(r->id, std::move(r));
  }
  s->cv_work.notify_all();
  return LV_OK;
}

lv_status lv_server_submit(lv_server* s, int64_t n, const int64_t* row_ptr, const int32_t* col,
                           const float* w, int64_t* request_id) {
  return server_submit(s, n, row_ptr, col, w, false, request_id);
}

lv_status lv_server_submit_borrowed(lv_server* s, int64_t n, const int64_t* row_ptr,
                                    const int32_t* col, const float* w, int64_t* request_id) {
  return server_submit(s, n, row_ptr, col, w, true, request_id);
}

lv_status lv_server_progress(lv_server* s, int64_t* n_done, int64_t* n_inflight, int64_t* n_queued) {
  if (!s) return LV_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  if (n_done) *n_done = s->n_done;
  if (n_inflight) *n_inflight = s->n_running;
  if (n_queued) *n_queued = (int64_t)s->queue.size();
  return LV_OK;
}

lv_status lv_server_poll(lv_server* s, int64_t request_id, int32_t* out_comm, double* out_modularity,
                         double* latency_ms, int32_t* done) {
  if (!s || !done) return LV_ERR_ARGUMENT;
  std::unique_ptr<lv::Request> r;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return LV_ERR_ARGUMENT;
    if (it->second->state != 2) {
      *done = 0;
      return LV_OK;
    }
    r = std::move(it->second);
    s->all.erase(it);
  }
  *done = 1;
  if (latency_ms)
    *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  if (r->status != LV_OK) {
    if (s->ctx) s->ctx->err = r->err;
    return r->status;
  }
  if (out_comm) std::memcpy(out_comm, r->out.data(), r->out.size() * 4);
  if (out_modularity) *out_modularity = r->modularity;
  return LV_OK;
}

lv_status lv_server_drain(lv_server* s) {
  if (!s) return LV_ERR_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->queue.empty() && s->n_running == 0; });
  return LV_OK;
}

}  // extern "C"
