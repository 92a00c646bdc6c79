// serving.cu -- request loop with continuous batching over resident
// references (b200d2_server_*).  No counterpart in the reference harness,
// which scores one particle file at a time (src/main.cu:483-503).
//
// Requests are queued by submit() and admitted by one scheduler thread: a
// request starts as soon as a stream slot is free and its device footprint
// (inputs, outputs, workspace) fits the HBM budget, in arrival order with
// later requests allowed past one that does not fit yet.  An admitted request
// runs entirely on its slot's stream, in the slot's device buffer (kept
// between requests, grown in the slot stream's order): host-to-device copies,
// the batch pipeline, device-to-host copies, and an end event that the
// scheduler polls to complete the request.  Requests on different slots
// overlap on the GPU.  The scheduler thread never waits for the GPU: host
// buffers that are not page-locked (a copy to or from them would block the
// issuing thread until the stream reaches it) go through the slot's
// page-locked staging buffer, inputs copied into it on the host before the
// upload, outputs copied out of it when the request completes.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

struct Ref {
  b200d2_view view;
  std::vector<float> eulers;  // [O_all][9]
  int O_all, N_img;
};

// A host-to-host copy the completion callback makes (staged output -> the
// caller's buffer).
struct HostCopy {
  void* dst;
  const void* src;
  size_t bytes;
};

struct Req {
  long long ticket = 0;
  b200d2_request r{};
  std::vector<float> eul;  // gathered [O][9]
  std::vector<HostCopy> out_copies;
  size_t ws_bytes = 0, footprint = 0;
  int status = -1;  // -1 pending, else a b200d2_status
  double t_submit = 0, t_done = 0, device_s = 0, t_admit = 0;
  int slot = -1;
  void* dbuf = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;  // both events recorded on the slot stream
  bool polled = false;  // completion found by the scheduler polling ev1 (no host callback)
  std::atomic<int> finished{0};
  struct b200d2_server* srv = nullptr;
  // a merged admission: the other requests its run carries (this one holds
  // the slot, the footprint, the events and the completion callback); a
  // member is finished by the scheduler when its leader is
  std::vector<std::shared_ptr<Req>> members;
  bool member = false;
};

}  // namespace

struct b200d2_server {
  int slots = 1;
  size_t budget = 0;
  int prec = B200D2_PREC_TF32;
  int device = 0;
  std::vector<Ref> refs;
  std::vector<cudaStream_t> streams;
  std::vector<int> slot_busy;
  cudaMemPool_t pool = nullptr;    // device memory of the slots
  std::vector<void*> dev;          // per slot: device buffer of its request, grown on its own stream
  std::vector<size_t> dev_bytes;
  std::vector<void*> pin;          // per slot: page-locked staging buffer
  std::vector<size_t> pin_bytes;
  std::vector<void*> pin_retired;  // outgrown staging buffers, freed with the server
  std::deque<std::shared_ptr<Req>> queue;
  std::vector<std::shared_ptr<Req>> inflight;
  std::map<long long, std::shared_ptr<Req>> all;
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::thread sched;
  bool stop = false;
  long long next_ticket = 1;
  b200d2_server_stats st{};
  // merged admissions (b200d2_server_set_merging): queued requests on one
  // reference run as one batch, at most this many requests and particles
  int merge_requests = 8, merge_particles = 512;
  int merge_request_particles = 128;  // only requests this small are merged
};

namespace {

void CUDART_CB on_done(void* arg) {
  Req* q = static_cast<Req*>(arg);
  for (const HostCopy& c : q->out_copies) memcpy(c.dst, c.src, c.bytes);
  q->t_done = now_s();
  q->finished.store(1);
  q->srv->cv_sched.notify_all();
}

// How an admitted request's completion is found.  With its end event
// recorded, the scheduler thread polls that event (it wakes every 200 us):
// a host callback (cudaLaunchHostFunc) runs on the one thread CUDA keeps for
// the callbacks of all streams, and at a light load completions reached
// through it came up to 27 ms after the work ended.  Without the event, a
// host callback marks the completion.
int finish_on(cudaStream_t st, Req& q) {
  if (q.timed) {
    q.polled = true;
    return B200D2_OK;
  }
  const cudaError_t e = cudaLaunchHostFunc(st, on_done, &q);
  if (e != cudaSuccess) return b200d2::status_from_cuda(e);
  return B200D2_OK;
}

// True when host memory at p is page-locked (or registered), so that an
// asynchronous copy from or to it does not block the calling thread.
bool page_locked(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // unregistered memory on older runtimes: clear the error
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// The slot's staging buffer, at least `need` bytes.  Called for an idle slot
// (its previous request's copies and callback have completed).
void* slot_staging(b200d2_server* s, int slot, size_t need) {
  if (need == 0) return nullptr;
  if (s->pin_bytes[slot] < need) {
    // cudaFreeHost waits for the device to go idle, which would stall every
    // slot: an outgrown buffer is kept until the server is destroyed
    if (s->pin[slot]) s->pin_retired.push_back(s->pin[slot]);
    s->pin[slot] = nullptr;
    s->pin_bytes[slot] = 0;
    const size_t bytes = std::max(need + need / 2, (size_t)1 << 20);
    if (cudaHostAlloc(&s->pin[slot], bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      s->pin[slot] = nullptr;
      return nullptr;
    }
    s->pin_bytes[slot] = bytes;
  }
  return s->pin[slot];
}

// The slot's device buffer, at least `need` bytes.  Called for an idle slot
// before its next request's work is issued on its stream, so a replacement
// is freed and allocated in that stream's order (no other stream ever waits
// on it).  Sizes are powers of two from 32 MiB (within the budget), so a slot
// grows a few times at most; when growing would take the slots' buffers past
// the budget, the buffers of idle slots are released first.
void* slot_device(b200d2_server* s, int slot, size_t need) {
  if (s->dev_bytes[slot] >= need) return s->dev[slot];
  size_t want = (size_t)32 << 20;
  while (want < need) want <<= 1;
  if (want > s->budget) want = need;
  need = want;
  cudaStream_t st = s->streams[slot];
  if (s->dev[slot]) cudaFreeAsync(s->dev[slot], st);
  s->dev[slot] = nullptr;
  s->dev_bytes[slot] = 0;
  size_t held = 0;
  for (size_t b : s->dev_bytes) held += b;
  for (int k = 0; k < s->slots && held + need > s->budget; ++k)
    if (k != slot && !s->slot_busy[k] && s->dev[k]) {
      cudaFreeAsync(s->dev[k], s->streams[k]);
      held -= s->dev_bytes[k];
      s->dev[k] = nullptr;
      s->dev_bytes[k] = 0;
    }
  if (cudaMallocFromPoolAsync(&s->dev[slot], need, s->pool, st) != cudaSuccess) {
    cudaGetLastError();
    s->dev[slot] = nullptr;
    return nullptr;
  }
  s->dev_bytes[slot] = need;
  return s->dev[slot];
}

// Launch a request's work on its slot stream (called with the lock held).
int admit(b200d2_server* s, Req& q) {
  char label[64];
  snprintf(label, sizeof(label), "b200d2 request %lld (ref %d, %d particles)", q.ticket, q.r.ref, q.r.P);
  b200d2::NvtxRange range(label);
  const Ref& ref = s->refs[q.r.ref];
  cudaStream_t st = s->streams[q.slot];
  const b200d2_request& r = q.r;
  const size_t img = (size_t)r.P * ref.N_img * sizeof(float);
  const size_t out = (size_t)r.P * r.O * r.T * sizeof(float);
  size_t off = 0;
  auto take = [&](size_t b) {
    size_t a = off;
    off += up256(b);
    return a;
  };
  const size_t o_re = take(img), o_im = take(img), o_co = take(img), o_eu = take((size_t)r.O * 9 * sizeof(float)),
               o_tx = take((size_t)r.T * sizeof(float)), o_ty = take((size_t)r.T * sizeof(float)),
               o_out = take(out), o_mn = take((size_t)r.P * sizeof(double)),
               o_am = take((size_t)r.P * sizeof(long long)), o_ws = take(q.ws_bytes);
  (void)o_ws;
  // host side: which buffers go through the staging buffer, and where
  struct Up {
    size_t dev_off;
    const void* src;
    size_t bytes;
    bool staged;
    size_t pin_off;
  };
  struct Down {
    void* dst;
    size_t dev_off;
    size_t bytes;
    bool staged;
    size_t pin_off;
  };
  size_t pin_need = 0;
  auto stage_at = [&](size_t bytes) {
    size_t a = pin_need;
    pin_need += up256(bytes);
    return a;
  };
  Up ups[6] = {{o_re, r.h_real, img, false, 0},
               {o_im, r.h_imag, img, false, 0},
               {o_co, r.h_corr, img, false, 0},
               {o_eu, q.eul.data(), q.eul.size() * sizeof(float), true, 0},
               {o_tx, r.h_trans_x, (size_t)r.T * sizeof(float), false, 0},
               {o_ty, r.h_trans_y, (size_t)r.T * sizeof(float), false, 0}};
  for (Up& u : ups) {
    if (!u.staged) u.staged = !page_locked(u.src);
    if (u.staged) u.pin_off = stage_at(u.bytes);
  }
  Down downs[3] = {{r.h_diff2, o_out, out, false, 0},
                   {r.h_min, o_mn, (size_t)r.P * sizeof(double), false, 0},
                   {r.h_argmin, o_am, (size_t)r.P * sizeof(long long), false, 0}};
  for (Down& w : downs) {
    if (!w.dst) continue;
    w.staged = !page_locked(w.dst);
    if (w.staged) w.pin_off = stage_at(w.bytes);
  }
  // a failed call leaves its error as this thread's last error, which the
  // next launch check would report: start every request from a clean state
  cudaGetLastError();
  uint8_t* pin = static_cast<uint8_t*>(slot_staging(s, q.slot, pin_need));
  if (pin_need && !pin) return B200D2_ERR_OOM;
  q.out_copies.clear();
  const double t_grow = now_s();
  q.dbuf = slot_device(s, q.slot, q.footprint);
  s->st.admit_grow_max_s = std::max(s->st.admit_grow_max_s, now_s() - t_grow);
  if (!q.dbuf) return B200D2_ERR_OOM;
  uint8_t* d = static_cast<uint8_t*>(q.dbuf);
  // the first failure among the copies and event records; the request still
  // runs to its completion callback and reports it
  cudaError_t first = cudaSuccess;
  auto note = [&](cudaError_t e) {
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  };
  note(cudaEventRecord(q.ev0, st));
  for (const Up& u : ups) {
    const void* src = u.src;
    if (u.staged) {
      memcpy(pin + u.pin_off, u.src, u.bytes);
      src = pin + u.pin_off;
    }
    note(cudaMemcpyAsync(d + u.dev_off, src, u.bytes, cudaMemcpyHostToDevice, st));
  }
  b200d2_batch b;
  memset(&b, 0, sizeof(b));
  b.d_eulers = reinterpret_cast<const float*>(d + o_eu);
  b.O = r.O;
  b.d_trans_x = reinterpret_cast<const float*>(d + o_tx);
  b.d_trans_y = reinterpret_cast<const float*>(d + o_ty);
  b.T = r.T;
  b.P = r.P;
  b.N_img = ref.N_img;
  b.d_real = reinterpret_cast<const float*>(d + o_re);
  b.d_imag = reinterpret_cast<const float*>(d + o_im);
  b.d_corr = reinterpret_cast<const float*>(d + o_co);
  b.img_stride = ref.N_img;
  b.d_diff2 = reinterpret_cast<float*>(d + o_out);
  b.accumulate = 0;
  b.d_min = reinterpret_cast<double*>(d + o_mn);
  b.d_argmin = reinterpret_cast<long long*>(d + o_am);
  const double t_run = now_s();
  int rc = b200d2_diff2_coarse_batch(&ref.view, &b, s->prec, q.ws_bytes ? d + o_ws : nullptr, q.ws_bytes, st);
  s->st.admit_launch_max_s = std::max(s->st.admit_launch_max_s, now_s() - t_run);
  for (const Down& w : downs) {
    if (!w.dst) continue;
    if (w.staged) {
      note(cudaMemcpyAsync(pin + w.pin_off, d + w.dev_off, w.bytes, cudaMemcpyDeviceToHost, st));
      q.out_copies.push_back(HostCopy{w.dst, pin + w.pin_off, w.bytes});
    } else {
      note(cudaMemcpyAsync(w.dst, d + w.dev_off, w.bytes, cudaMemcpyDeviceToHost, st));
    }
  }
  note(cudaEventRecord(q.ev1, st));
  q.timed = first == cudaSuccess;
  if (rc == B200D2_OK && first != cudaSuccess) rc = b200d2::status_from_cuda(first);
  q.status = rc;  // final status once finished
  return finish_on(st, q);
}

// A merged admission: requests on one reference (arrival order, the first
// one the leader) as one block-diagonal batch.  Each request's orientations
// take columns from a multiple of 256, so that no tile of the contraction
// holds two requests' columns.
struct MergedLayout {
  std::vector<b200d2::MergedRequest> mr;
  int O_cols = 0, P = 0;
  b200d2::MergedBatch* mb = nullptr;
  size_t footprint = 0;
};

int merged_layout(b200d2_server* s, const std::vector<std::shared_ptr<Req>>& grp, MergedLayout& L) {
  const Ref& ref = s->refs[grp[0]->r.ref];
  L.mr.clear();
  L.P = 0;
  long long col = 0;
  for (const auto& q : grp) {
    b200d2::MergedRequest m;
    m.P = q->r.P;
    m.O = q->r.O;
    m.T = q->r.T;
    m.col0 = (int)col;
    m.h_tx = q->r.h_trans_x;
    m.h_ty = q->r.h_trans_y;
    L.mr.push_back(m);
    col = (col + q->r.O + 255) / 256 * 256;
    L.P += q->r.P;
  }
  if (col > (1 << 30)) return B200D2_ERR_TOO_LARGE;
  L.O_cols = L.mr.back().col0 + L.mr.back().O;
  int st = B200D2_OK;
  L.mb = b200d2::merged_create(ref.view, ref.N_img, s->prec, L.mr.data(), (int)L.mr.size(), L.O_cols, &st);
  if (!L.mb) return st;
  size_t fp = up256((size_t)L.O_cols * 9 * sizeof(float)) + up256((size_t)L.P * sizeof(double)) +
              up256((size_t)L.P * sizeof(long long)) + up256(b200d2::merged_device_bytes(L.mb));
  for (const auto& q : grp)
    fp += 3 * up256((size_t)q->r.P * ref.N_img * sizeof(float)) +
          up256((size_t)q->r.P * q->r.O * q->r.T * sizeof(float));
  L.footprint = fp;
  return B200D2_OK;
}

// Launch a merged admission's work on the leader's slot stream (called with
// the lock held): every request's copies in, one pipeline run, every
// request's copies out, one completion callback.
int admit_merged(b200d2_server* s, Req& lead, const std::vector<std::shared_ptr<Req>>& grp, MergedLayout& L) {
  char label[80];
  snprintf(label, sizeof(label), "b200d2 merged requests %lld.. (%d requests, ref %d, %d particles)", lead.ticket,
           (int)grp.size(), lead.r.ref, L.P);
  b200d2::NvtxRange range(label);
  const Ref& ref = s->refs[lead.r.ref];
  cudaStream_t st = s->streams[lead.slot];
  const int n = (int)grp.size();
  size_t off = 0;
  auto take = [&](size_t b) {
    size_t a = off;
    off += up256(b);
    return a;
  };
  struct Up {
    size_t dev_off;
    const void* src;
    size_t bytes;
    bool staged;
    size_t pin_off;
  };
  struct Down {
    void* dst;
    size_t dev_off;
    size_t bytes;
    bool staged;
    size_t pin_off;
  };
  size_t pin_need = 0;
  auto stage_at = [&](size_t bytes) {
    size_t a = pin_need;
    pin_need += up256(bytes);
    return a;
  };
  // staging: the batch's tables first (256-byte aligned), the merged
  // orientations, then the host buffers that are not page-locked
  const size_t p_tab = stage_at(b200d2::merged_host_bytes(L.mb));
  const size_t eu_bytes = (size_t)L.O_cols * 9 * sizeof(float);
  const size_t p_eu = stage_at(eu_bytes);
  const size_t o_eu = take(eu_bytes), o_mn = take((size_t)L.P * sizeof(double)),
               o_am = take((size_t)L.P * sizeof(long long));
  std::vector<b200d2::MergedDev> md(n);
  std::vector<size_t> o_in(n), o_out(n);
  std::vector<Up> ups;
  std::vector<Down> downs;
  int part0 = 0;
  for (int k = 0; k < n; ++k) {
    const b200d2_request& r = grp[k]->r;
    const size_t img = (size_t)r.P * ref.N_img * sizeof(float);
    const size_t out = (size_t)r.P * r.O * r.T * sizeof(float);
    o_in[k] = take(img);
    take(img);
    take(img);
    o_out[k] = take(out);
    ups.push_back({o_in[k], r.h_real, img, false, 0});
    ups.push_back({o_in[k] + up256(img), r.h_imag, img, false, 0});
    ups.push_back({o_in[k] + 2 * up256(img), r.h_corr, img, false, 0});
    if (r.h_diff2) downs.push_back({r.h_diff2, o_out[k], out, false, 0});
    if (r.h_min) downs.push_back({r.h_min, o_mn + (size_t)part0 * sizeof(double), (size_t)r.P * sizeof(double), false, 0});
    if (r.h_argmin)
      downs.push_back({r.h_argmin, o_am + (size_t)part0 * sizeof(long long), (size_t)r.P * sizeof(long long), false, 0});
    part0 += r.P;
  }
  const size_t o_mb = take(b200d2::merged_device_bytes(L.mb));
  for (Up& u : ups) {
    u.staged = !page_locked(u.src);
    if (u.staged) u.pin_off = stage_at(u.bytes);
  }
  for (Down& w : downs) {
    w.staged = !page_locked(w.dst);
    if (w.staged) w.pin_off = stage_at(w.bytes);
  }
  cudaGetLastError();  // start from a clean error state (see admit)
  uint8_t* pin = static_cast<uint8_t*>(slot_staging(s, lead.slot, pin_need));
  if (!pin) return B200D2_ERR_OOM;
  lead.out_copies.clear();
  const double t_grow = now_s();
  lead.dbuf = slot_device(s, lead.slot, lead.footprint);
  s->st.admit_grow_max_s = std::max(s->st.admit_grow_max_s, now_s() - t_grow);
  if (!lead.dbuf) return B200D2_ERR_OOM;
  uint8_t* d = static_cast<uint8_t*>(lead.dbuf);
  // the merged orientations: each request's Euler matrices at its columns;
  // the columns between requests (projected, read by no particle) repeat the
  // next request's first matrix
  float* eu = reinterpret_cast<float*>(pin + p_eu);
  int end = 0;
  for (int k = 0; k < n; ++k) {
    const b200d2::MergedRequest& m = L.mr[k];
    for (int c = end; c < m.col0; ++c) memcpy(eu + (size_t)c * 9, grp[k]->eul.data(), 9 * sizeof(float));
    memcpy(eu + (size_t)m.col0 * 9, grp[k]->eul.data(), (size_t)m.O * 9 * sizeof(float));
    end = m.col0 + m.O;
  }
  cudaError_t first = cudaSuccess;
  auto note = [&](cudaError_t e) {
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  };
  note(cudaEventRecord(lead.ev0, st));
  for (const Up& u : ups) {
    const void* src = u.src;
    if (u.staged) {
      memcpy(pin + u.pin_off, u.src, u.bytes);
      src = pin + u.pin_off;
    }
    note(cudaMemcpyAsync(d + u.dev_off, src, u.bytes, cudaMemcpyHostToDevice, st));
  }
  note(cudaMemcpyAsync(d + o_eu, eu, eu_bytes, cudaMemcpyHostToDevice, st));
  for (int k = 0; k < n; ++k) {
    const size_t img = up256((size_t)grp[k]->r.P * ref.N_img * sizeof(float));
    md[k].re = reinterpret_cast<const float*>(d + o_in[k]);
    md[k].im = reinterpret_cast<const float*>(d + o_in[k] + img);
    md[k].corr = reinterpret_cast<const float*>(d + o_in[k] + 2 * img);
    md[k].out = reinterpret_cast<float*>(d + o_out[k]);
  }
  const double t_run = now_s();
  int rc = b200d2::merged_enqueue(L.mb, reinterpret_cast<const float*>(d + o_eu), md.data(),
                                  reinterpret_cast<double*>(d + o_mn), reinterpret_cast<long long*>(d + o_am),
                                  d + o_mb, pin + p_tab, st);
  s->st.admit_launch_max_s = std::max(s->st.admit_launch_max_s, now_s() - t_run);
  for (const Down& w : downs) {
    if (w.staged) {
      note(cudaMemcpyAsync(pin + w.pin_off, d + w.dev_off, w.bytes, cudaMemcpyDeviceToHost, st));
      lead.out_copies.push_back(HostCopy{w.dst, pin + w.pin_off, w.bytes});
    } else {
      note(cudaMemcpyAsync(w.dst, d + w.dev_off, w.bytes, cudaMemcpyDeviceToHost, st));
    }
  }
  note(cudaEventRecord(lead.ev1, st));
  lead.timed = first == cudaSuccess;
  if (rc == B200D2_OK && first != cudaSuccess) rc = b200d2::status_from_cuda(first);
  lead.status = rc;
  return finish_on(st, lead);
}

void sched_loop(b200d2_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    for (size_t i = 0; i < s->inflight.size();) {
      Req& q = *s->inflight[i];
      if (q.polled && !q.finished.load()) {
        const cudaError_t e = cudaEventQuery(q.ev1);
        if (e == cudaSuccess) {
          on_done(&q);
        } else if (e != cudaErrorNotReady) {
          cudaGetLastError();
          q.status = b200d2::status_from_cuda(e);
          q.t_done = now_s();
          q.finished.store(1);
        }
      }
      if (q.finished.load()) {
        // a request that failed before its work was issued has no recorded
        // events (asking for their elapsed time would fail and leave an error)
        float ms = 0.f;
        if (q.timed && cudaEventElapsedTime(&ms, q.ev0, q.ev1) == cudaSuccess) q.device_s = ms / 1e3;
        cudaGetLastError();
        if (q.status == -1) q.status = B200D2_OK;
        if (q.timed) {
          // where a request's latency went: waiting for admission, and the
          // time from admission to its completion callback beyond its stream time
          s->st.queue_wait_max_s = std::max(s->st.queue_wait_max_s, q.t_admit - q.t_submit);
          s->st.done_lag_max_s = std::max(s->st.done_lag_max_s, q.t_done - q.t_admit - q.device_s);
          for (const std::shared_ptr<Req>& m : q.members)
            s->st.queue_wait_max_s = std::max(s->st.queue_wait_max_s, q.t_admit - m->t_submit);
        }
        s->slot_busy[q.slot] = 0;
        s->st.bytes_in_use -= q.footprint;
        s->st.stream_s += q.device_s;
        s->st.completed++;
        if (q.status == B200D2_OK) s->st.evals += (long long)q.r.P * q.r.O * q.r.T;
        // the requests merged into this one's run finish with it
        for (const std::shared_ptr<Req>& m : q.members) {
          m->device_s = q.device_s;
          m->t_done = q.t_done;
          m->status = q.status;
          s->st.completed++;
          if (m->status == B200D2_OK) s->st.evals += (long long)m->r.P * m->r.O * m->r.T;
          m->finished.store(1);
        }
        q.members.clear();
        s->inflight.erase(s->inflight.begin() + i);
        progress = true;
      } else {
        ++i;
      }
    }
    if (progress) s->cv_done.notify_all();
    for (auto it = s->queue.begin(); it != s->queue.end();) {
      Req& q = **it;
      // an idle slot whose buffer already holds the request (the smallest
      // such), else the idle slot with the largest buffer, which grows: a
      // growth maps new memory while the scheduler waits, so it is avoided
      // whenever an idle slot can take the request as it is
      int slot = -1, fit = -1;
      for (int k = 0; k < s->slots; ++k) {
        if (s->slot_busy[k]) continue;
        if (s->dev_bytes[k] >= q.footprint && (fit < 0 || s->dev_bytes[k] < s->dev_bytes[fit])) fit = k;
        if (slot < 0 || s->dev_bytes[k] > s->dev_bytes[slot]) slot = k;
      }
      if (slot < 0) break;
      if (fit >= 0) slot = fit;
      if (s->st.bytes_in_use + q.footprint > s->budget) {
        ++it;
        continue;
      }
      // under a backlog (more queued requests than idle slots), merge later
      // queued requests on the same reference into this one's run while the
      // particle and request limits and the budget allow, and while the
      // merged run fits an idle slot's buffer as it is (a merge never makes a
      // slot grow, which maps memory while the queue waits).  Without a
      // backlog every request gets a slot of its own: merging then would put
      // work on one slot that idle slots could run beside it.
      const double t_merge = now_s();  // the merge decision counts as admission time
      std::vector<std::shared_ptr<Req>> grp;
      MergedLayout L;
      size_t idle_max = 0;
      int idle = 0;
      for (int k = 0; k < s->slots; ++k)
        if (!s->slot_busy[k]) {
          idle_max = std::max(idle_max, s->dev_bytes[k]);
          ++idle;
        }
      // Only small requests are merged: a large one fills the GPU with its
      // own pipeline, and bundling it would hold the others until it ends.
      const int small = std::min(s->merge_request_particles, s->merge_particles);
      if (s->merge_requests > 1 && b200d2::is_tc_precision(s->prec) && q.r.P <= small &&
          q.footprint < idle_max && (int)s->queue.size() > idle) {
        grp.push_back(*it);
        int P = q.r.P;
        for (auto jt = std::next(it); jt != s->queue.end() && (int)grp.size() < s->merge_requests; ++jt)
          if ((*jt)->r.ref == q.r.ref && (*jt)->r.P <= small && P + (*jt)->r.P <= s->merge_particles) {
            grp.push_back(*jt);
            P += (*jt)->r.P;
          }
        // a group that does not fit is halved (its tables are built once per try)
        while (grp.size() > 1) {
          if (merged_layout(s, grp, L) == B200D2_OK && s->st.bytes_in_use + L.footprint <= s->budget &&
              L.footprint <= idle_max)
            break;
          b200d2::merged_destroy(L.mb);
          L.mb = nullptr;
          grp.resize(grp.size() / 2);
        }
        if (grp.size() < 2) grp.clear();
      }
      if (!grp.empty()) {
        // the slot for the merged footprint, chosen as above
        int fit2 = -1;
        for (int k = 0; k < s->slots; ++k)
          if (!s->slot_busy[k] && s->dev_bytes[k] >= L.footprint && (fit2 < 0 || s->dev_bytes[k] < s->dev_bytes[fit2]))
            fit2 = k;
        if (fit2 >= 0) {
          slot = fit2;
        } else {
          for (int k = 0; k < s->slots; ++k)
            if (!s->slot_busy[k] && s->dev_bytes[k] > s->dev_bytes[slot]) slot = k;
        }
        q.slot = slot;
        q.footprint = L.footprint;
        s->slot_busy[slot] = 1;
        s->st.bytes_in_use += q.footprint;
        s->st.peak_bytes = std::max(s->st.peak_bytes, s->st.bytes_in_use);
        for (size_t k = 1; k < grp.size(); ++k) {
          grp[k]->member = true;
          grp[k]->footprint = 0;
          q.members.push_back(grp[k]);
        }
        const double t_admit = now_s();
        q.t_admit = t_admit;
        const int rc = admit_merged(s, q, grp, L);
        s->st.admit_host_s += now_s() - t_admit;
        s->st.admit_host_max_s = std::max(s->st.admit_host_max_s, now_s() - t_merge);
        b200d2::merged_destroy(L.mb);
        if (rc != B200D2_OK && !q.finished.load()) {
          q.status = rc;
          q.t_done = now_s();
          q.finished.store(1);
        }
        s->st.merged_admissions++;
        s->st.merged_requests += (long long)grp.size();
        s->inflight.push_back(*it);
        s->queue.erase(std::remove_if(s->queue.begin(), s->queue.end(),
                                      [&](const std::shared_ptr<Req>& x) {
                                        return x.get() == &q || x->member;
                                      }),
                       s->queue.end());
        int busy = 0;
        for (const auto& x : s->inflight) busy += 1 + (int)x->members.size();
        s->st.max_in_flight = std::max(s->st.max_in_flight, busy);
        progress = true;
        it = s->queue.begin();  // the queue changed: scan it again
        continue;
      }
      q.slot = slot;
      s->slot_busy[slot] = 1;
      s->st.bytes_in_use += q.footprint;
      s->st.peak_bytes = std::max(s->st.peak_bytes, s->st.bytes_in_use);
      const double t_admit = now_s();
      q.t_admit = t_admit;
      const int rc = admit(s, q);
      s->st.admit_host_s += now_s() - t_admit;
      s->st.admit_host_max_s = std::max(s->st.admit_host_max_s, now_s() - t_admit);
      if (rc != B200D2_OK && !q.finished.load()) {
        // nothing was left on the stream that would signal completion
        q.status = rc;
        q.t_done = now_s();
        q.finished.store(1);
      }
      s->inflight.push_back(*it);
      it = s->queue.erase(it);
      int busy = 0;
      for (const auto& x : s->inflight) busy += 1 + (int)x->members.size();
      s->st.max_in_flight = std::max(s->st.max_in_flight, busy);
      progress = true;
    }
    {
      int busy = 0;
      for (const auto& x : s->inflight) busy += 1 + (int)x->members.size();
      s->st.in_flight = busy;
    }
    s->st.queued = (int)s->queue.size();
    if (s->stop && s->queue.empty() && s->inflight.empty()) break;
    if (!progress) s->cv_sched.wait_for(lk, std::chrono::microseconds(200));
  }
}

}  // namespace

extern "C" int b200d2_server_create(int slots, size_t hbm_budget_bytes, int precision, b200d2_server** out) {
  if (!out || slots <= 0 || slots > 64 || hbm_budget_bytes == 0) return B200D2_ERR_INVALID;
  if (precision != B200D2_PREC_FP32 && !b200d2::is_tc_precision(precision))
    return B200D2_ERR_UNSUPPORTED;
  *out = nullptr;
  b200d2_server* s = new b200d2_server();
  s->slots = slots;
  s->budget = hbm_budget_bytes;
  s->prec = precision;
  cudaGetDevice(&s->device);
  s->slot_busy.assign(slots, 0);
  s->pin.assign(slots, nullptr);
  s->pin_bytes.assign(slots, 0);
  s->dev.assign(slots, nullptr);
  s->dev_bytes.assign(slots, 0);
  for (int k = 0; k < slots; ++k) {
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
      delete s;
      return B200D2_ERR_CUDA;
    }
    s->streams.push_back(st);
  }
  // the server's own memory pool for the slots' buffers: no internal
  // dependencies, so memory released by one slot never makes another slot's
  // stream wait (it is reused once its free has completed)
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->device;
  if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
    for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
    delete s;
    return B200D2_ERR_CUDA;
  }
  uint64_t thr = hbm_budget_bytes;
  int no = 0, yes = 1;
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowOpportunistic, &yes);
  // map the first part of the budget (up to 8 GiB) now, so that the slots'
  // buffers are carved from memory the pool already holds instead of mapping
  // new memory (milliseconds per growth) while requests wait
  {
    void* warm = nullptr;
    const size_t reserve = std::min(hbm_budget_bytes, (size_t)8 << 30);
    if (cudaMallocFromPoolAsync(&warm, reserve, s->pool, s->streams[0]) == cudaSuccess) {
      cudaFreeAsync(warm, s->streams[0]);
      cudaStreamSynchronize(s->streams[0]);
    } else {
      cudaGetLastError();
    }
  }
  // load every kernel the requests can launch now: a kernel loaded at its
  // first launch (lazy module loading) can wait for the slots' running work
  if (b200d2::is_tc_precision(precision) && b200d2::tc_preload(precision) != B200D2_OK) cudaGetLastError();
  // page-locked staging buffers of a first size, so that small requests and
  // merged tables do not pin memory while the queue waits
  for (int k = 0; k < slots; ++k) slot_staging(s, k, (size_t)8 << 20);
  cudaGetLastError();
  s->sched = std::thread(sched_loop, s);
  *out = s;
  return B200D2_OK;
}

extern "C" int b200d2_server_add_reference(b200d2_server* s, const b200d2_view* view, const float* h_eulers,
                                           int O_all, int N_img, int* ref_id) {
  if (!s || !view || !h_eulers || O_all <= 0 || N_img <= 0 || !ref_id) return B200D2_ERR_INVALID;
  if ((long long)view->imgX * view->imgY < N_img) return B200D2_ERR_INVALID;
  Ref r;
  r.view = *view;
  r.eulers.assign(h_eulers, h_eulers + (size_t)O_all * 9);
  r.O_all = O_all;
  r.N_img = N_img;
  std::lock_guard<std::mutex> lk(s->mu);
  s->refs.push_back(std::move(r));
  *ref_id = (int)s->refs.size() - 1;
  return B200D2_OK;
}

extern "C" int b200d2_server_submit(b200d2_server* s, const b200d2_request* req, long long* ticket) {
  if (!s || !req || !ticket) return B200D2_ERR_INVALID;
  const b200d2_request& r = *req;
  if (r.P <= 0 || r.O <= 0 || r.T <= 0 || !r.h_real || !r.h_imag || !r.h_corr || !r.h_orient || !r.h_trans_x ||
      !r.h_trans_y)
    return B200D2_ERR_INVALID;
  auto q = std::make_shared<Req>();
  q->r = r;
  q->srv = s;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (r.ref < 0 || r.ref >= (int)s->refs.size()) return B200D2_ERR_INVALID;
    const Ref& ref = s->refs[r.ref];
    q->eul.resize((size_t)r.O * 9);
    for (int k = 0; k < r.O; ++k) {
      const int o = r.h_orient[k];
      if (o < 0 || o >= ref.O_all) return B200D2_ERR_INVALID;
      memcpy(&q->eul[(size_t)k * 9], &ref.eulers[(size_t)o * 9], 9 * sizeof(float));
    }
    // workspace of this shape (the size query needs only non-null pointers)
    b200d2_batch b;
    memset(&b, 0, sizeof(b));
    const float* dummy = reinterpret_cast<const float*>(256);
    b.d_eulers = b.d_trans_x = b.d_trans_y = b.d_real = b.d_imag = b.d_corr = dummy;
    b.d_diff2 = const_cast<float*>(dummy);
    b.O = r.O;
    b.T = r.T;
    b.P = r.P;
    b.N_img = ref.N_img;
    b.img_stride = ref.N_img;
    q->ws_bytes = b200d2_diff2_coarse_batch_workspace(&ref.view, &b, s->prec);
    const size_t img = up256((size_t)r.P * ref.N_img * sizeof(float));
    q->footprint = 3 * img + up256((size_t)r.O * 9 * sizeof(float)) + 2 * up256((size_t)r.T * sizeof(float)) +
                   up256((size_t)r.P * r.O * r.T * sizeof(float)) + up256((size_t)r.P * sizeof(double)) +
                   up256((size_t)r.P * sizeof(long long)) + up256(q->ws_bytes);
    s->st.submitted++;
    if (q->footprint > s->budget) {
      s->st.rejected++;
      return B200D2_ERR_TOO_LARGE;
    }
    if (cudaEventCreate(&q->ev0) != cudaSuccess || cudaEventCreate(&q->ev1) != cudaSuccess) return B200D2_ERR_CUDA;
    q->ticket = s->next_ticket++;
    q->t_submit = now_s();
    s->all[q->ticket] = q;
    s->queue.push_back(q);
    *ticket = q->ticket;
  }
  s->cv_sched.notify_all();
  return B200D2_OK;
}

extern "C" int b200d2_server_wait(b200d2_server* s, long long ticket, double timeout_s, double* latency_s,
                                  double* device_s) {
  if (!s) return B200D2_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return B200D2_ERR_INVALID;
  std::shared_ptr<Req> q = it->second;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (!(q->finished.load() && std::find(s->inflight.begin(), s->inflight.end(), q) == s->inflight.end() &&
           std::find(s->queue.begin(), s->queue.end(), q) == s->queue.end())) {
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) return B200D2_ERR_TIMEOUT;
  }
  if (latency_s) *latency_s = q->t_done - q->t_submit;
  if (device_s) *device_s = q->device_s;
  const int status = q->status;
  cudaEventDestroy(q->ev0);
  cudaEventDestroy(q->ev1);
  q->ev0 = q->ev1 = nullptr;
  s->all.erase(it);
  return status;
}

extern "C" int b200d2_server_cancel(b200d2_server* s, long long ticket) {
  if (!s) return B200D2_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return B200D2_ERR_INVALID;
    if (it->second->status == B200D2_ERR_CANCELLED) return B200D2_OK;  // cancelled before
    auto qi = std::find(s->queue.begin(), s->queue.end(), it->second);
    if (qi == s->queue.end()) return B200D2_ERR_UNSUPPORTED;  // admitted already
    Req& q = **qi;
    q.status = B200D2_ERR_CANCELLED;
    q.t_done = now_s();
    q.finished.store(1);
    s->queue.erase(qi);
    s->st.cancelled++;
    s->st.queued = (int)s->queue.size();
  }
  s->cv_done.notify_all();
  s->cv_sched.notify_all();
  return B200D2_OK;
}

extern "C" int b200d2_server_set_merging(b200d2_server* s, int max_requests, int max_particles,
                                         int max_request_particles) {
  if (!s || max_requests < 1 || max_particles < 1 || max_request_particles < 1) return B200D2_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  s->merge_requests = max_requests;
  s->merge_particles = max_particles;
  s->merge_request_particles = max_request_particles;
  return B200D2_OK;
}

extern "C" int b200d2_server_get_stats(b200d2_server* s, b200d2_server_stats* st) {
  if (!s || !st) return B200D2_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->st;
  // the maxima cover the time since the previous read
  s->st.admit_host_max_s = s->st.admit_grow_max_s = s->st.admit_launch_max_s = 0.0;
  s->st.queue_wait_max_s = s->st.done_lag_max_s = 0.0;
  return B200D2_OK;
}

extern "C" int b200d2_server_destroy(b200d2_server* s) {
  if (!s) return B200D2_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_sched.notify_all();
  if (s->sched.joinable()) s->sched.join();
  for (cudaStream_t x : s->streams) {
    cudaStreamSynchronize(x);
    cudaStreamDestroy(x);
  }
  for (void* p : s->pin)
    if (p) cudaFreeHost(p);
  for (void* p : s->pin_retired) cudaFreeHost(p);
  for (void* p : s->dev)
    if (p) cudaFree(p);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  for (auto& kv : s->all) {
    if (kv.second->ev0) cudaEventDestroy(kv.second->ev0);
    if (kv.second->ev1) cudaEventDestroy(kv.second->ev1);
  }
  delete s;
  return B200D2_OK;
}
