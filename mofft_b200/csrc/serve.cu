// Serving loop: continuous batching of FFT requests on one GPU (host code).
//
// A worker thread owns the GPU side.  It admits pending requests in arrival
// order while their payload bytes fit the HBM budget, takes with the head
// request every other pending request of the same (length, precision,
// direction) -- whatever has arrived by then, up to max_group_points -- and
// runs the group as ONE indirect batched launch on a free stream: host
// payloads are staged into pooled device memory, a table of per-transform
// device pointers is uploaded, the plan's passes run over the table, results
// are copied back, and an event recorded behind the work marks the group.
// A lone request on device buffers skips the table and runs as a plain
// batched launch.  Up to `streams` groups are in flight, so copies and
// kernels of different groups overlap and new arrivals wait at most for one
// stream and enough memory.  While groups are in flight the worker polls
// their events every few microseconds (no host callback thread in the
// completion path).
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/mofft_serve.h"
#include "mofft_host.h"

namespace {

struct Req {
  mofft_request r;
  uint64_t ticket = 0;
  double t_submit = 0.0, t_done = 0.0;
  mofft_status status = MOFFT_SUCCESS;
  bool done = false;
  bool host_in = false, host_out = false;
  size_t payload = 0;   // input + output bytes
};

// A staging block from the pool.
struct Block {
  void *ptr = nullptr;
  size_t cls = 0;
};

struct Stream {
  cudaStream_t s = nullptr;
  cudaEvent_t done = nullptr;  // recorded behind the group's work
  bool busy = false;
  bool recorded = false;       // `done` covers the current group
  std::vector<Req *> group;
  std::vector<Block> blocks;
  size_t admitted = 0;
  void **h_table = nullptr;   // pinned host pointer table
  void **d_table = nullptr;
  size_t table_cap = 0;       // entries per direction (in and out)
};

using PlanKey = std::tuple<size_t, int, int>;

}  // namespace

struct mofft_server {
  mofft_server_options opt{};
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work;
  std::condition_variable cv_done;
  std::deque<Req *> pending;
  std::unordered_map<uint64_t, Req *> reqs;
  uint64_t next_ticket = 1;
  std::vector<Stream> streams;
  std::map<PlanKey, mofft_core *> plans;
  std::map<size_t, std::vector<void *>> pool;   // worker thread only
  size_t admitted = 0;
  mofft_server_stats stats{};
  bool stop = false;
  std::thread worker;
};

namespace {

size_t elem_bytes(int bits) { return bits == 32 ? 8 : 16; }

bool pool_get(mofft_server *S, size_t bytes, Block *b) {
  size_t cls = size_t(1) << 20;
  while (cls < bytes) cls <<= 1;
  b->cls = cls;
  std::vector<void *> &v = S->pool[cls];
  if (!v.empty()) {
    b->ptr = v.back();
    v.pop_back();
    return true;
  }
  if (cudaMalloc(&b->ptr, cls) != cudaSuccess) {
    cudaGetLastError();
    b->ptr = nullptr;
    return false;
  }
  return true;
}

void pool_put(mofft_server *S, const Block &b) {
  if (b.ptr) S->pool[b.cls].push_back(b.ptr);
}

mofft_core *plan_for(mofft_server *S, const mofft_request &r, mofft_status *st) {
  const PlanKey key(r.length, r.precision_bits, (int)r.direction);
  auto it = S->plans.find(key);
  if (it != S->plans.end()) {
    *st = MOFFT_SUCCESS;
    return it->second;
  }
  // the tuned schedule (compiled wisdom) where one exists; the model's where
  // the tuned one has more passes than a pointer-table group runs (two)
  mofft_core *c = nullptr;
  *st = mofft_core_create_pretuned(&c, r.precision_bits, r.length, 1, 0, r.direction,
                                   MOFFT_OUT_OF_PLACE);
  if (*st == MOFFT_SUCCESS && c->sched.pass_count > 2) {
    mofft_core_destroy(c);
    c = nullptr;
    *st = mofft_core_create(&c, r.precision_bits, r.length, 1, 0, r.direction,
                            MOFFT_OUT_OF_PLACE, nullptr, 0);
  }
  if (*st != MOFFT_SUCCESS) return nullptr;
  S->plans[key] = c;
  return c;
}

// Issue one group on stream `idx` (worker thread, no lock held).
mofft_status launch_group(mofft_server *S, int idx) {
  Stream &st = S->streams[idx];
  const mofft_request &head = st.group.front()->r;
  mofft_status status;
  mofft_core *plan = plan_for(S, head, &status);
  if (!plan) return status;
  const size_t eb = elem_bytes(head.precision_bits);
  const size_t n = head.length;
  const bool two_pass = plan->sched.pass_count > 1;
  // Runtime-stage (generic) kernels take no pointer tables: such a group runs
  // one plain batched launch per request on the same stream.
  bool tables = true;
  for (int p = 0; p < plan->sched.pass_count; ++p)
    if (plan->sched.pass[p].kind != MOFFT_KERNEL_ROWS &&
        plan->sched.pass[p].kind != MOFFT_KERNEL_COLS)
      tables = false;
  if (!tables && plan->sched.pass_count > 2) return MOFFT_UNSUPPORTED_SIZE;
  if (st.group.size() == 1) {
    const Req *q = st.group.front();
    const bool in_place = q->r.input == q->r.output;
    if (!q->host_in && !q->host_out && !(in_place && two_pass) &&
        plan->sched.pass_count <= 2) {
      status = mofft_core_enqueue_batch(plan, q->r.input, q->r.output, q->r.batch, n, st.s);
      if (status != MOFFT_SUCCESS) return status;
      if (cudaEventRecord(st.done, st.s) != cudaSuccess) return MOFFT_INTERNAL_ERROR;
      return MOFFT_SUCCESS;
    }
  }
  size_t transforms = 0;
  for (Req *q : st.group) transforms += q->r.batch;
  if (transforms > st.table_cap) {
    if (st.h_table) cudaFreeHost(st.h_table);
    if (st.d_table) cudaFree(st.d_table);
    st.h_table = nullptr;
    st.d_table = nullptr;
    size_t cap = 1024;
    while (cap < transforms) cap <<= 1;
    if (cudaHostAlloc(reinterpret_cast<void **>(&st.h_table), 2 * cap * sizeof(void *),
                      cudaHostAllocDefault) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&st.d_table), 2 * cap * sizeof(void *)) !=
            cudaSuccess) {
      cudaGetLastError();
      st.table_cap = 0;
      return MOFFT_ALLOCATION_FAILURE;
    }
    st.table_cap = cap;
  }
  struct Post {
    void *dst;
    const void *src;
    size_t bytes;
    cudaMemcpyKind kind;
  };
  std::vector<Post> post;
  size_t k = 0;
  for (Req *q : st.group) {
    const size_t bytes = q->r.batch * n * eb;
    const unsigned char *din = static_cast<const unsigned char *>(q->r.input);
    unsigned char *dout = static_cast<unsigned char *>(q->r.output);
    const bool in_place = q->r.input == q->r.output;
    if (q->host_in) {
      Block b;
      if (!pool_get(S, bytes, &b)) return MOFFT_ALLOCATION_FAILURE;
      st.blocks.push_back(b);
      if (cudaMemcpyAsync(b.ptr, q->r.input, bytes, cudaMemcpyHostToDevice, st.s) != cudaSuccess)
        return MOFFT_INTERNAL_ERROR;
      din = static_cast<const unsigned char *>(b.ptr);
    }
    // outputs that cannot be written directly: host buffers, and in-place
    // requests of two-pass lengths (the first pass may not overwrite its input)
    if (q->host_out || (in_place && two_pass)) {
      Block b;
      if (!pool_get(S, bytes, &b)) return MOFFT_ALLOCATION_FAILURE;
      st.blocks.push_back(b);
      post.push_back({q->r.output, b.ptr, bytes,
                      q->host_out ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice});
      dout = static_cast<unsigned char *>(b.ptr);
    }
    if (!tables) {
      status = mofft_core_enqueue_batch(plan, din, dout, q->r.batch, n, st.s);
      if (status != MOFFT_SUCCESS) return status;
      continue;
    }
    for (size_t t = 0; t < q->r.batch; ++t, ++k) {
      st.h_table[k] = const_cast<unsigned char *>(din) + t * n * eb;
      st.h_table[st.table_cap + k] = dout + t * n * eb;
    }
  }
  if (tables) {
    if (cudaMemcpyAsync(st.d_table, st.h_table, k * sizeof(void *), cudaMemcpyHostToDevice,
                        st.s) != cudaSuccess ||
        cudaMemcpyAsync(st.d_table + st.table_cap, st.h_table + st.table_cap,
                        k * sizeof(void *), cudaMemcpyHostToDevice, st.s) != cudaSuccess)
      return MOFFT_INTERNAL_ERROR;
    status = mofft_core_enqueue_indirect(plan, st.d_table, st.d_table + st.table_cap,
                                         (long long)transforms, st.s);
    if (status != MOFFT_SUCCESS) return status;
  }
  for (const Post &p : post)
    if (cudaMemcpyAsync(p.dst, p.src, p.bytes, p.kind, st.s) != cudaSuccess)
      return MOFFT_INTERNAL_ERROR;
  if (cudaEventRecord(st.done, st.s) != cudaSuccess) return MOFFT_INTERNAL_ERROR;
  return MOFFT_SUCCESS;
}

// Lock held.  Marks the group of stream idx complete with `status`.
void finish_group(mofft_server *S, int idx, mofft_status status, double t_done) {
  Stream &st = S->streams[idx];
  for (Req *q : st.group) {
    q->status = status;
    q->t_done = t_done;
    q->done = true;
    if (status == MOFFT_SUCCESS) ++S->stats.completed;
    else ++S->stats.failed;
  }
  for (const Block &b : st.blocks) pool_put(S, b);
  st.blocks.clear();
  st.group.clear();
  S->admitted -= st.admitted;
  st.admitted = 0;
  st.busy = false;
  st.recorded = false;
  S->cv_done.notify_all();
}

int free_stream(mofft_server *S) {
  for (size_t i = 0; i < S->streams.size(); ++i)
    if (!S->streams[i].busy) return (int)i;
  return -1;
}

bool same_key(const mofft_request &a, const mofft_request &b) {
  return a.length == b.length && a.precision_bits == b.precision_bits &&
         a.direction == b.direction;
}

// Lock held.  Moves the next group from `pending` to stream idx; returns
// false if the head request must wait for memory.
bool form_group(mofft_server *S, int idx) {
  Stream &st = S->streams[idx];
  while (!S->pending.empty()) {
    Req *head = S->pending.front();
    if (S->admitted + head->payload > S->opt.hbm_budget_bytes) {
      if (S->admitted == 0) {   // can never fit
        S->pending.pop_front();
        head->status = MOFFT_ALLOCATION_FAILURE;
        head->done = true;
        head->t_done = mofft_monotonic_seconds();
        ++S->stats.failed;
        S->cv_done.notify_all();
        continue;
      }
      return false;
    }
    size_t points = head->r.batch * head->r.length;
    size_t bytes = head->payload;
    st.group.push_back(head);
    std::deque<Req *> rest;
    S->pending.pop_front();
    while (!S->pending.empty()) {
      Req *q = S->pending.front();
      S->pending.pop_front();
      const size_t qp = q->r.batch * q->r.length;
      if (same_key(q->r, head->r) && points + qp <= S->opt.max_group_points &&
          S->admitted + bytes + q->payload <= S->opt.hbm_budget_bytes) {
        st.group.push_back(q);
        points += qp;
        bytes += q->payload;
      } else {
        rest.push_back(q);
      }
    }
    S->pending.swap(rest);
    st.admitted = bytes;
    S->admitted += bytes;
    if (S->admitted > S->stats.peak_admitted_bytes) S->stats.peak_admitted_bytes = S->admitted;
    st.busy = true;
    st.recorded = false;
    return true;
  }
  return false;
}

void worker_main(mofft_server *S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lock(S->mu);
  for (;;) {
    for (size_t i = 0; i < S->streams.size(); ++i) {
      Stream &st = S->streams[i];
      if (!st.busy || !st.recorded) continue;
      const cudaError_t q = cudaEventQuery(st.done);
      if (q == cudaSuccess) {
        finish_group(S, (int)i, MOFFT_SUCCESS, mofft_monotonic_seconds());
      } else if (q != cudaErrorNotReady) {
        cudaGetLastError();
        finish_group(S, (int)i, MOFFT_INTERNAL_ERROR, mofft_monotonic_seconds());
      }
    }
    int idx;
    while ((idx = free_stream(S)) >= 0 && form_group(S, idx)) {
      lock.unlock();
      const mofft_status st = launch_group(S, idx);
      lock.lock();
      ++S->stats.launches;
      if (st == MOFFT_SUCCESS) S->streams[idx].recorded = true;
      if (st != MOFFT_SUCCESS) {
        // wait for whatever was already enqueued on the stream, then fail
        lock.unlock();
        cudaStreamSynchronize(S->streams[idx].s);
        cudaGetLastError();
        lock.lock();
        finish_group(S, idx, st, mofft_monotonic_seconds());
      }
    }
    bool busy = false;
    for (const Stream &s : S->streams) busy |= s.busy;
    if (S->stop && S->pending.empty() && !busy) break;
    auto startable = [&] {
      if (S->stop) return true;
      if (S->pending.empty()) return false;
      if (free_stream(S) < 0) return false;
      return S->admitted + S->pending.front()->payload <= S->opt.hbm_budget_bytes ||
             S->admitted == 0;
    };
    if (busy)   // poll the in-flight groups' events
      S->cv_work.wait_for(lock, std::chrono::microseconds(10), startable);
    else
      S->cv_work.wait(lock, startable);
  }
}

bool is_device(const void *p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" mofft_status mofft_server_create(mofft_server **out,
                                            const mofft_server_options *options) {
  if (!out) return MOFFT_INVALID_ARGUMENT;
  *out = nullptr;
  if (!mofft_hardware_supports(32)) return MOFFT_UNSUPPORTED_HARDWARE;
  mofft_server *S = new (std::nothrow) mofft_server();
  if (!S) return MOFFT_ALLOCATION_FAILURE;
  if (options) S->opt = *options;
  if (S->opt.hbm_budget_bytes == 0) S->opt.hbm_budget_bytes = size_t(40) << 30;
  if (S->opt.streams <= 0) S->opt.streams = 4;
  if (S->opt.streams > 64) S->opt.streams = 64;
  if (S->opt.max_group_points == 0) S->opt.max_group_points = size_t(1) << 27;
  cudaGetDevice(&S->device);
  S->streams.resize((size_t)S->opt.streams);
  for (int i = 0; i < S->opt.streams; ++i) {
    if (cudaStreamCreateWithFlags(&S->streams[i].s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->streams[i].done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      mofft_server_destroy(S);
      return MOFFT_INTERNAL_ERROR;
    }
  }
  S->worker = std::thread(worker_main, S);
  *out = S;
  return MOFFT_SUCCESS;
}

extern "C" mofft_status mofft_server_submit(mofft_server *S, const mofft_request *r,
                                            uint64_t *ticket) {
  if (!S || !r || !ticket || !r->input || !r->output || r->batch == 0 || r->length < 2 ||
      (r->direction != MOFFT_FORWARD && r->direction != MOFFT_BACKWARD) ||
      (r->precision_bits != 32 && r->precision_bits != 64))
    return MOFFT_INVALID_ARGUMENT;
  if (!mofft_is_smooth13(r->length)) return MOFFT_UNSUPPORTED_SIZE;
  Req *q = new (std::nothrow) Req();
  if (!q) return MOFFT_ALLOCATION_FAILURE;
  q->r = *r;
  q->host_in = !is_device(r->input);
  q->host_out = r->output == r->input ? q->host_in : !is_device(r->output);
  q->payload = 2 * r->batch * r->length * elem_bytes(r->precision_bits);
  q->t_submit = mofft_monotonic_seconds();
  std::lock_guard<std::mutex> lock(S->mu);
  q->ticket = S->next_ticket++;
  S->reqs[q->ticket] = q;
  S->pending.push_back(q);
  ++S->stats.submitted;
  *ticket = q->ticket;
  S->cv_work.notify_one();
  return MOFFT_SUCCESS;
}

extern "C" mofft_status mofft_server_wait(mofft_server *S, uint64_t ticket,
                                          double *latency_seconds) {
  if (!S) return MOFFT_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return MOFFT_INVALID_ARGUMENT;
  Req *q = it->second;
  S->cv_done.wait(lock, [&] { return q->done; });
  if (latency_seconds) *latency_seconds = q->t_done - q->t_submit;
  const mofft_status st = q->status;
  S->reqs.erase(it);
  delete q;
  return st;
}

extern "C" mofft_status mofft_server_drain(mofft_server *S) {
  if (!S) return MOFFT_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(S->mu);
  S->cv_done.wait(lock, [&] {
    return S->stats.completed + S->stats.failed == S->stats.submitted;
  });
  return MOFFT_SUCCESS;
}

extern "C" mofft_status mofft_server_get_stats(mofft_server *S, mofft_server_stats *stats) {
  if (!S || !stats) return MOFFT_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(S->mu);
  *stats = S->stats;
  return MOFFT_SUCCESS;
}

extern "C" void mofft_server_destroy(mofft_server *S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    S->stop = true;
    S->cv_work.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  for (Stream &st : S->streams) {
    if (st.s) cudaStreamSynchronize(st.s);
    if (st.h_table) cudaFreeHost(st.h_table);
    if (st.d_table) cudaFree(st.d_table);
    if (st.done) cudaEventDestroy(st.done);
    if (st.s) cudaStreamDestroy(st.s);
  }
  for (auto &kv : S->pool)
    for (void *p : kv.second) cudaFree(p);
  for (auto &kv : S->plans) mofft_core_destroy(kv.second);
  for (auto &kv : S->reqs) delete kv.second;
  delete S;
}
