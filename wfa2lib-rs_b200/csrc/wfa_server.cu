// wfa_server.cu -- the serving loop: continuous batching of single requests
// over the batched C-ABI entry points (host code only).
//
// Submitters append requests to one of three lane queues (short, long
// high-memory, BiWFA).  Each worker thread serves one lane and owns an
// aligner handle (its own stream and device buffers); it repeatedly takes
// every waiting request of its lane that fits into a batch (in arrival
// order, up to max_batch_pairs and max_batch_bytes of predicted wavefront
// memory), runs it with wfa_batch_align (end-to-end, or the BiWFA span) and
// files the results for pollers.  Several batches are on the GPU at once,
// short requests never queue behind long batches, and a request that
// arrives while batches run joins the next batch a worker of its lane forms.
//
// With `resident` set, the short lane is a resident stream instead
// (wfa_stream_*: a persistent kernel that takes requests as they come): a
// collector thread moves its results to the finished list, and a short
// request that finds the stream's ring full takes the batch lane.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/wfa_b200.h"

namespace wfab {
int preload_kernels(int device);  // wfa_capi.cu
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id;
  std::vector<uint8_t> seq;  // pattern then text
  int32_t n, m;
  int64_t pred;  // predicted wavefront bytes in its mode
  int32_t mode;  // 0 high memory, 1 BiWFA
  Clock::time_point t0;
};

struct Finished {
  wfa_served_t rec;
  std::vector<uint8_t> cigar;
};

// Predicted wavefront memory of a pair: the M history of high memory holds
// O(s^2) cells with s about (n + m) / 4, i.e. about (n + m)^2 / 4 bytes; BiWFA
// holds two rings of scope x components x (n + m) cells (26 x 5 for the
// two-piece affine scope of the default penalties).
int64_t predict_high(int64_t len) { return len * len / 4; }
int64_t predict_biwfa(int64_t len) { return 2 * 26 * 5 * 4 * (len + 3); }

}  // namespace

struct wfa_server {
  wfa_server_config_t cfg{};
  std::mutex mu;
  std::condition_variable cv_work[3], cv_done;
  std::deque<Request> queue[3];  // lanes: 0 short, 1 long high memory, 2 BiWFA
  std::deque<Finished> done;
  std::vector<std::thread> threads;
  std::vector<wfa_aligner_t*> handles;
  std::vector<int> lane_of;  // per worker
  bool stopping = false;
  int64_t next_id = 0;
  int64_t outstanding = 0;  // submitted and not yet polled
  std::string last_error;   // of the last failed batch
  // Resident short lane: the stream, its requests (stream id -> server id,
  // submit time), the collector thread.
  wfa_stream_t* stream = nullptr;
  std::map<int64_t, std::pair<int64_t, Clock::time_point>> in_stream;
  std::thread collector;

  void run_batch(wfa_aligner_t* h, std::vector<Request>& reqs, int span);
  void worker(int w);
  void collect();
};

void wfa_server::collect() {
  std::vector<wfa_served_t> recs(4096);
  std::vector<uint8_t> cig((size_t)4096 * (2 * (size_t)cfg.short_max_len + 1));
  for (;;) {
    const int32_t c = wfa_stream_poll(stream, recs.data(), (int32_t)recs.size(), cig.data(),
                                      (int64_t)cig.size(), 2);
    const Clock::time_point t1 = Clock::now();
    std::lock_guard<std::mutex> lock(mu);
    if (c < 0) {
      // The stream failed: its outstanding requests carry the error code.
      last_error = "resident stream failed";
      for (auto& kv : in_stream) {
        Finished f;
        std::memset(&f.rec, 0, sizeof f.rec);
        f.rec.id = kv.second.first;
        f.rec.status = c;
        f.rec.cigar_offset = -1;
        done.push_back(std::move(f));
      }
      in_stream.clear();
      cv_done.notify_all();
      return;
    }
    for (int32_t j = 0; j < c; ++j) {
      const wfa_served_t& r = recs[(size_t)j];
      auto it = in_stream.find(r.id);
      if (it == in_stream.end()) continue;
      Finished f;
      f.rec = r;
      f.rec.id = it->second.first;
      f.rec.cigar_offset = -1;
      f.rec.latency_ns = std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - it->second.second).count();
      if (r.cigar_length > 0) f.cigar.assign(cig.begin() + r.cigar_offset, cig.begin() + r.cigar_offset + r.cigar_length);
      in_stream.erase(it);
      done.push_back(std::move(f));
    }
    if (c > 0) cv_done.notify_all();
    if (stopping && in_stream.empty()) return;
  }
}

void wfa_server::run_batch(wfa_aligner_t* h, std::vector<Request>& reqs, int span) {
  if (reqs.empty()) return;
  const int64_t k = (int64_t)reqs.size();
  std::vector<int64_t> po((size_t)k), to((size_t)k);
  std::vector<int32_t> pl((size_t)k), tl((size_t)k);
  int64_t bytes = 0, cig_cap = 0;
  for (const Request& r : reqs) {
    bytes += (int64_t)r.seq.size();
    cig_cap += 2 * ((int64_t)r.n + r.m) + 1;
  }
  std::vector<uint8_t> seq((size_t)bytes + 16, 0);
  int64_t at = 0;
  for (int64_t i = 0; i < k; ++i) {
    const Request& r = reqs[(size_t)i];
    std::memcpy(seq.data() + at, r.seq.data(), r.seq.size());
    po[(size_t)i] = at;
    pl[(size_t)i] = r.n;
    to[(size_t)i] = at + r.n;
    tl[(size_t)i] = r.m;
    at += (int64_t)r.seq.size();
  }
  std::vector<wfa_result_t> res((size_t)k);
  std::vector<uint8_t> cig((size_t)cig_cap + 16);
  wfa_batch_t b{};
  b.format = WFA_SEQ_ASCII;
  b.span = span;
  b.num_pairs = k;
  b.seq = seq.data();
  b.seq_bytes = bytes;
  b.p_off = po.data();
  b.p_len = pl.data();
  b.t_off = to.data();
  b.t_len = tl.data();
  const int rc = wfa_batch_align(h, &b, res.data(), cfg.score_only ? nullptr : cig.data());
  const Clock::time_point t1 = Clock::now();
  if (rc != WFA_OK) {
    std::lock_guard<std::mutex> lock(mu);
    last_error = wfa_last_error_string(h);
  }
  std::vector<Finished> out((size_t)k);
  for (int64_t i = 0; i < k; ++i) {
    const Request& r = reqs[(size_t)i];
    Finished& f = out[(size_t)i];
    std::memset(&f.rec, 0, sizeof f.rec);
    f.rec.id = r.id;
    f.rec.mode = r.mode;
    f.rec.cigar_offset = -1;
    f.rec.latency_ns = std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - r.t0).count();
    if (rc != WFA_OK) {
      f.rec.status = rc;  // the batch's error code
      continue;
    }
    const wfa_result_t& x = res[(size_t)i];
    f.rec.score = x.score;
    f.rec.status = x.status;
    f.rec.cigar_length = x.cigar_length;
    f.rec.cigar_score = x.cigar_score;
    f.rec.end_v = x.end_v;
    f.rec.end_h = x.end_h;
    if (!cfg.score_only && x.cigar_length > 0)
      f.cigar.assign(cig.begin() + x.cigar_begin, cig.begin() + x.cigar_begin + x.cigar_length);
  }
  {
    std::lock_guard<std::mutex> lock(mu);
    for (Finished& f : out) done.push_back(std::move(f));
  }
  cv_done.notify_all();
}

void wfa_server::worker(int w) {
  cudaSetDevice(cfg.device);
  wfa_aligner_t* h = handles[(size_t)w];
  const int lane = lane_of[(size_t)w];
  std::deque<Request>& q = queue[lane];
  for (;;) {
    std::vector<Request> batch;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_work[lane].wait(lock, [&] { return stopping || !q.empty(); });
      if (q.empty()) return;  // stopping, nothing left
      int64_t bytes = 0, count = 0;
      while (!q.empty() && count < cfg.max_batch_pairs) {
        Request& r = q.front();
        if (count > 0 && bytes + r.pred > cfg.max_batch_bytes) break;
        bytes += r.pred;
        ++count;
        batch.push_back(std::move(r));
        q.pop_front();
      }
      if (!q.empty()) cv_work[lane].notify_one();
    }
    run_batch(h, batch, lane == 2 ? WFA_SPAN_BIWFA : WFA_SPAN_END2END);
  }
}

extern "C" {

wfa_server_t* wfa_server_start(const wfa_server_config_t* config, int* err) {
  if (!config) {
    if (err) *err = WFA_ERR_ARGUMENT;
    return nullptr;
  }
  wfa_server_t* s = new wfa_server();
  s->cfg = *config;
  if (s->cfg.workers <= 0) s->cfg.workers = 2;
  if (s->cfg.short_workers <= 0) s->cfg.short_workers = 2;
  if (s->cfg.biwfa_workers <= 0) s->cfg.biwfa_workers = 2;
  if (s->cfg.short_max_len <= 0) s->cfg.short_max_len = 1024;
  if (s->cfg.max_batch_pairs <= 0) s->cfg.max_batch_pairs = 65536;
  if (s->cfg.max_batch_bytes <= 0) s->cfg.max_batch_bytes = 4ll << 30;
  if (s->cfg.biwfa_above_bytes <= 0) s->cfg.biwfa_above_bytes = 256ll << 20;
  const int counts[3] = {s->cfg.short_workers, s->cfg.workers, s->cfg.biwfa_workers};
  for (int lane = 0; lane < 3; ++lane)
    for (int i = 0; i < counts[lane]; ++i) s->lane_of.push_back(lane);
  for (size_t w = 0; w < s->lane_of.size(); ++w) {
    int e = WFA_OK;
    wfa_aligner_t* h = wfa_aligner_create((wfa_metric_t)s->cfg.metric, &s->cfg.penalties,
                                          s->cfg.device, &e);
    if (!h) {
      for (wfa_aligner_t* x : s->handles) wfa_aligner_destroy(x);
      delete s;
      if (err) *err = e;
      return nullptr;
    }
    wfa_set_alignment_scope(h, s->cfg.score_only ? WFA_SCOPE_SCORE : WFA_SCOPE_ALIGNMENT);
    s->handles.push_back(h);
  }
  if (s->cfg.resident) {
    // The resident short lane holds one block per SM, so that the batch
    // lanes' kernels find room beside it; every kernel is loaded before it
    // starts (a first launch beside it would wait for it to end).
    int e = wfab::preload_kernels(s->cfg.device);
    if (e != WFA_OK) {
      for (wfa_aligner_t* x : s->handles) wfa_aligner_destroy(x);
      delete s;
      if (err) *err = e;
      return nullptr;
    }
    s->stream = wfa_stream_start((wfa_metric_t)s->cfg.metric, &s->cfg.penalties, s->cfg.device, s->cfg.score_only,
                                 std::min(s->cfg.short_max_len, 2048), 1 << 16, 1, &e);
    if (!s->stream) {
      for (wfa_aligner_t* x : s->handles) wfa_aligner_destroy(x);
      delete s;
      if (err) *err = e;
      return nullptr;
    }
    s->collector = std::thread(&wfa_server::collect, s);
  }
  for (size_t w = 0; w < s->lane_of.size(); ++w) s->threads.emplace_back(&wfa_server::worker, s, (int)w);
  if (err) *err = WFA_OK;
  return s;
}

int64_t wfa_server_submit(wfa_server_t* s, const uint8_t* pattern, int32_t n, const uint8_t* text,
                          int32_t m) {
  if (!s || n < 0 || m < 0 || (n > 0 && !pattern) || (m > 0 && !text)) return WFA_ERR_ARGUMENT;
  Request r;
  r.seq.resize((size_t)n + (size_t)m);
  if (n) std::memcpy(r.seq.data(), pattern, (size_t)n);
  if (m) std::memcpy(r.seq.data() + n, text, (size_t)m);
  r.n = n;
  r.m = m;
  const int64_t len = (int64_t)n + m;
  const int64_t high = predict_high(len);
  r.mode = high > s->cfg.biwfa_above_bytes ? 1 : 0;
  r.pred = r.mode ? predict_biwfa(len) : high;
  const int lane = r.mode ? 2 : (len <= s->cfg.short_max_len ? 0 : 1);
  r.t0 = Clock::now();
  int64_t id;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) return WFA_ERR_ARGUMENT;
    id = r.id = s->next_id++;
    ++s->outstanding;
    if (lane == 0 && s->stream) {
      const int64_t sid = wfa_stream_submit(s->stream, pattern, n, text, m);
      if (sid >= 0) {
        s->in_stream[sid] = std::make_pair(id, r.t0);
        return id;
      }
      // ring full (or the stream failed): the batch lane takes it
    }
    s->queue[lane].push_back(std::move(r));
  }
  s->cv_work[lane].notify_one();
  return id;
}

int32_t wfa_server_poll(wfa_server_t* s, wfa_served_t* out, int32_t max, uint8_t* cigars,
                        int64_t cigar_cap, int32_t timeout_ms) {
  if (!s || !out || max <= 0) return WFA_ERR_ARGUMENT;
  std::unique_lock<std::mutex> lock(s->mu);
  if (s->done.empty() && timeout_ms > 0)
    s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty(); });
  int32_t c = 0;
  int64_t used = 0;
  while (c < max && !s->done.empty()) {
    Finished& f = s->done.front();
    const int64_t len = (int64_t)f.cigar.size();
    if (len > 0) {
      if (!cigars || used + len > cigar_cap) {
        if (c == 0) return WFA_ERR_ARGUMENT;  // the next CIGAR does not fit the buffer
        break;
      }
      std::memcpy(cigars + used, f.cigar.data(), (size_t)len);
      f.rec.cigar_offset = used;
      used += len;
    }
    out[c++] = f.rec;
    s->done.pop_front();
    --s->outstanding;
  }
  return c;
}

const char* wfa_server_last_error(wfa_server_t* s) {
  if (!s) return "";
  std::lock_guard<std::mutex> lock(s->mu);
  return s->last_error.c_str();
}

int64_t wfa_server_pending(wfa_server_t* s) {
  if (!s) return WFA_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  return s->outstanding;
}

int wfa_server_stop(wfa_server_t* s) {
  if (!s) return WFA_ERR_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  for (auto& cv : s->cv_work) cv.notify_all();
  for (std::thread& t : s->threads) t.join();
  if (s->stream) {
    s->collector.join();
    wfa_stream_stop(s->stream);
  }
  for (wfa_aligner_t* h : s->handles) wfa_aligner_destroy(h);
  delete s;
  return WFA_OK;
}

}  // extern "C"
