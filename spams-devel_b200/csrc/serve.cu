// Serving loop: coding requests against dictionaries kept resident on one GPU.
//
// No counterpart in the reference (each SPAMS call is synchronous and brings
// its own dictionary).  A server holds, per dictionary id, D, its Gram
// matrices (DᵀD for OMP, DᵀD + 1e-10 I for the Lasso, as decomp/decomp.h:1569
// forms them with lambda2 = 0) and its three-piece BF16 split.  `slots` worker
// threads each own a CUDA stream and workspaces (a private DeviceCtx): a free
// slot takes the oldest pending request, merges every pending request with the
// same dictionary and options into one launch (serve_plan.h), admits it
// against the device-memory budget, copies the signals in, codes them with
// per-signal L / eps / lambda, and splits the CSC back per request.  Slots run
// concurrently, so requests that arrive while others are on the GPU start as
// soon as a slot and memory are free.  A signal's code never depends on the
// other signals of its launch (every kernel of the pipeline is per column).
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "kernels.h"
#include "serve_plan.h"

namespace sc {
namespace {

using Clock = std::chrono::steady_clock;

struct SrvDict {
  int64_t id = 0;
  int m = 0, K = 0, Kp = 0, mp = 0;
  Buf D, Gomp, Glasso, split;
  Buf GompTc, GlassoTc, tcerr;  // the Grams of the BF16x3 form (tensor cores)
  size_t bytes = 0;
  int users = 0;  // pending requests and batches in flight
};

struct SrvReq {
  int64_t ticket = 0;
  sc_request r{};
  PlanKey key;
  int Leff = 0;              // clamped L of this request
  Clock::time_point t0;      // arrival (scheduled arrival for replays)
  bool done = false;
  sc_status status = SC_OK;
  std::string err;
  double lat_ms = 0;
  int64_t* colptr = nullptr;
  int32_t* rows = nullptr;
  float* vals = nullptr;
  int64_t nnz = 0;
  void free_result() {
    free(colptr); free(rows); free(vals);
    colptr = nullptr; rows = nullptr; vals = nullptr;
  }
};

struct Slot {
  DeviceCtx* ctx = nullptr;
  std::thread th;
  Buf X, vecs, ocol, orows, ovals;
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  size_t reserved = 0;      // device bytes this slot's workspaces hold
  bool busy = false;
  sc_status host_buffer(size_t bytes) {
    if (bytes <= pinned_bytes) return SC_OK;
    const size_t want = std::max(bytes, pinned_bytes * 3 / 2);
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    pinned_bytes = 0;
    SC_CUDA(cudaHostAlloc(&pinned, want, cudaHostAllocDefault));
    pinned_bytes = want;
    return SC_OK;
  }
};

}  // namespace
}  // namespace sc

using namespace sc;

struct sc_server {
  int device = 0;
  size_t budget = 0;
  int64_t max_batch = 0;
  DeviceCtx* admin = nullptr;  // dictionary uploads
  std::mutex mu;
  std::condition_variable cv;       // slots: work or memory may be available
  std::condition_variable cv_done;  // waiters: a request completed
  std::map<int64_t, std::unique_ptr<SrvDict>> dicts;
  size_t dict_bytes = 0;
  size_t pool_warm = 0;  // bytes the stream-ordered pool was grown by for the slots
  std::deque<SrvReq*> pending;
  std::unordered_map<int64_t, SrvReq*> live;  // ticket -> request (until collected)
  std::vector<std::unique_ptr<Slot>> slots;
  int64_t next_ticket = 1;
  bool stop = false;
  // statistics (since the last reset)
  std::vector<double> lat;
  int64_t completed = 0, signals = 0, batches = 0, batch_reqs = 0, rejected = 0;
  std::string last_err;
  size_t peak = 0;
  int active = 0;
  Clock::time_point busy_from;
  double busy_s = 0;

  size_t reserved_total() const {
    size_t t = dict_bytes;
    for (auto& s : slots) t += s->reserved;
    return t;
  }
};

namespace {

void finish_request(sc_server* s, SrvReq* q, Clock::time_point now) {
  q->done = true;
  q->lat_ms = std::chrono::duration<double, std::milli>(now - q->t0).count();
  if (q->status == SC_OK) {
    s->lat.push_back(q->lat_ms);
    ++s->completed;
    s->signals += q->r.n;
  } else {
    ++s->rejected;
    s->last_err = q->err;
  }
  auto it = s->dicts.find(q->r.dict_id);
  if (it != s->dicts.end()) --it->second->users;
  if (q->r.flags & SC_REQ_DISCARD) {
    q->free_result();
    s->live.erase(q->ticket);
    delete q;
  }
}

// Codes one batch on slot `sl` (called without the server lock).
sc_status run_batch(sc_server* s, Slot& sl, SrvDict& d, std::vector<SrvReq*>& batch) {
  DeviceCtx& c = *sl.ctx;
  cudaStream_t st = c.stream;
  SC_CUDA(cudaSetDevice(s->device));
  // the slot's workspaces grow on its own stream (its previous batch has
  // completed), not through a device-wide synchronisation that would stall
  // the other slots
  AllocStream grow_on(st);
  const SrvReq& r0 = *batch.front();
  const bool lars = r0.r.algo == SC_REQ_LASSO;
  int64_t N = 0;
  int Lmax = 0;
  for (SrvReq* q : batch) {
    N += q->r.n;
    Lmax = std::max(Lmax, q->Leff);
  }
  const bool tc = r0.r.precision == SC_PREC_BF16X3;
  // signals in: one copy per request into consecutive columns
  SC_TRY(sl.X.reserve((size_t)d.m * N * 4));
  float* dX = reinterpret_cast<float*>(sl.X.ptr);
  {
    int64_t off = 0;
    for (SrvReq* q : batch) {
      SC_CUDA(cudaMemcpyAsync(dX + (size_t)off * d.m, q->r.X, (size_t)q->r.n * d.m * 4,
                              cudaMemcpyHostToDevice, st));
      off += q->r.n;
    }
  }
  // per-signal parameters: L (int), eps, lambda (OMP) or lambda1 (Lasso)
  const size_t vb = align16((size_t)N * 4);
  SC_TRY(sl.vecs.reserve(3 * vb));
  SC_TRY(sl.host_buffer(3 * vb + (size_t)(N + 1) * 8));
  char* hv = static_cast<char*>(sl.pinned);
  int* hL = reinterpret_cast<int*>(hv);
  float* hE = reinterpret_cast<float*>(hv + vb);
  float* hA = reinterpret_cast<float*>(hv + 2 * vb);
  {
    int64_t off = 0;
    for (SrvReq* q : batch) {
      for (int64_t i = 0; i < q->r.n; ++i) {
        hL[off + i] = q->Leff;
        hE[off + i] = q->r.eps;
        hA[off + i] = q->r.lambda1;
      }
      off += q->r.n;
    }
  }
  SC_CUDA(cudaMemcpyAsync(sl.vecs.ptr, hv, 3 * vb, cudaMemcpyHostToDevice, st));
  char* dv = static_cast<char*>(sl.vecs.ptr);
  // CSC out
  SC_TRY(sl.ocol.reserve((size_t)(N + 1) * 8));
  SC_TRY(sl.orows.reserve((size_t)N * Lmax * 4));
  SC_TRY(sl.ovals.reserve((size_t)N * Lmax * 4));

  BatchDesc b;
  b.lars = lars;
  b.dX = dX;
  b.m = d.m;
  b.n = N;
  b.dD = reinterpret_cast<const float*>(d.D.ptr);
  b.G = reinterpret_cast<const float*>(tc ? (lars ? d.GlassoTc.ptr : d.GompTc.ptr)
                                          : (lars ? d.Glasso.ptr : d.Gomp.ptr));
  b.dDsplit = tc ? d.split.ptr : nullptr;
  b.K = d.K;
  b.Kp = d.Kp;
  b.L = Lmax;
  b.tc = tc;
  b.refine = r0.r.refine > 0;
  if (lars) {
    b.mode = r0.r.mode;
    b.pos = r0.r.pos;
    b.length_path = r0.key.path;
    b.lambda1 = r0.r.lambda1;
    b.dLam1 = reinterpret_cast<const float*>(dv + 2 * vb);
  } else {
    b.Lsig = Lmax;
    b.dLv = reinterpret_cast<const int*>(dv);
    b.dEps = reinterpret_cast<const float*>(dv + vb);
    b.dLam = reinterpret_cast<const float*>(dv + 2 * vb);
  }
  b.d_colptr = reinterpret_cast<int64_t*>(sl.ocol.ptr);
  b.d_rows = reinterpret_cast<int32_t*>(sl.orows.ptr);
  b.d_vals = reinterpret_cast<float*>(sl.ovals.ptr);
  b.cap = N * (int64_t)Lmax;
  b.stream = st;
  SC_TRY(code_batch_f32(c, b));
  int64_t nnz = 0;
  SC_TRY(finish_batch(c, b, &nnz));
  // CSC back: colptr, then the entries of the requests that keep a result
  bool any_kept = false;
  for (SrvReq* q : batch) any_kept |= !(q->r.flags & SC_REQ_DISCARD);
  SC_TRY(sl.host_buffer((size_t)(N + 1) * 8 + (any_kept ? (size_t)nnz * 8 : 0)));
  int64_t* hcol = static_cast<int64_t*>(sl.pinned);
  int32_t* hrows = reinterpret_cast<int32_t*>(hcol + N + 1);
  float* hvals = reinterpret_cast<float*>(hrows + nnz);
  SC_CUDA(cudaMemcpyAsync(hcol, b.d_colptr, (size_t)(N + 1) * 8, cudaMemcpyDeviceToHost, st));
  if (any_kept && nnz > 0) {
    SC_CUDA(cudaMemcpyAsync(hrows, b.d_rows, (size_t)nnz * 4, cudaMemcpyDeviceToHost, st));
    SC_CUDA(cudaMemcpyAsync(hvals, b.d_vals, (size_t)nnz * 4, cudaMemcpyDeviceToHost, st));
  }
  SC_CUDA(cudaStreamSynchronize(st));
  int64_t off = 0;
  for (SrvReq* q : batch) {
    const int64_t n = q->r.n;
    const int64_t c0 = hcol[off], c1 = hcol[off + n];
    q->nnz = c1 - c0;
    if (!(q->r.flags & SC_REQ_DISCARD)) {
      q->colptr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
      q->rows = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(1, q->nnz));
      q->vals = (float*)malloc(sizeof(float) * (size_t)std::max<int64_t>(1, q->nnz));
      if (!q->colptr || !q->rows || !q->vals) {
        q->free_result();
        return fail(SC_ERR_OUT_OF_MEMORY, "host malloc failed");
      }
      for (int64_t i = 0; i <= n; ++i) q->colptr[i] = hcol[off + i] - c0;
      if (q->nnz > 0) {
        memcpy(q->rows, hrows + c0, sizeof(int32_t) * (size_t)q->nnz);
        memcpy(q->vals, hvals + c0, sizeof(float) * (size_t)q->nnz);
      }
    }
    off += n;
  }
  return SC_OK;
}

void slot_loop(sc_server* s, size_t idx) {
  Slot& sl = *s->slots[idx];
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<SrvReq*> batch;
    SrvDict* d = nullptr;
    size_t need = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->pending.empty()) {
          if (s->stop) return;
          s->cv.wait(lk);
          continue;
        }
        std::vector<PlanItem> items;
        items.reserve(s->pending.size());
        for (SrvReq* q : s->pending) items.push_back(PlanItem{q->key, q->r.n});
        std::vector<size_t> take = plan_batch(items, s->max_batch);
        SrvReq* q0 = s->pending[take[0]];
        d = s->dicts.at(q0->r.dict_id).get();
        int64_t N = 0;
        int Lmax = 0;
        for (size_t t : take) {
          N += s->pending[t]->r.n;
          Lmax = std::max(Lmax, s->pending[t]->Leff);
        }
        const bool tc = q0->r.precision == SC_PREC_BF16X3;
        need = batch_bytes(d->m, d->Kp, d->mp, Lmax, N, tc);
        // active sets beyond the shared-memory capacity rerun with global state
        // (at most 256 MiB, see the pipeline's overflow pass)
        if (Lmax > 32) need += (size_t)256 << 20;
        std::vector<size_t> res;
        for (auto& o : s->slots) res.push_back(o->reserved);
        if (!admit(s->dict_bytes, res, idx, need, s->budget)) {
          // idle slots give their workspaces back before anyone waits
          bool freed = false;
          for (size_t i = 0; i < s->slots.size(); ++i) {
            Slot& o = *s->slots[i];
            if (i != idx && !o.busy && o.reserved > 0) {
              destroy_ctx(o.ctx);
              o.ctx = nullptr;
              for (Buf* bb : {&o.X, &o.vecs, &o.ocol, &o.orows, &o.ovals}) bb->release();
              o.reserved = 0;
              freed = true;
            }
          }
          if (freed) continue;
          bool others_busy = false;
          for (size_t i = 0; i < s->slots.size(); ++i)
            others_busy |= i != idx && s->slots[i]->busy;
          if (!others_busy && sl.reserved > need) {
            // this slot's own high-water workspaces are in the way
            destroy_ctx(sl.ctx);
            sl.ctx = nullptr;
            for (Buf* bb : {&sl.X, &sl.vecs, &sl.ocol, &sl.orows, &sl.ovals}) bb->release();
            sl.reserved = 0;
            continue;
          }
          if (!others_busy) {
            // nothing in flight will free memory: the oldest request cannot run
            s->pending.erase(s->pending.begin() + (std::ptrdiff_t)take[0]);
            q0->status = SC_ERR_OUT_OF_MEMORY;
            q0->err = "serving: request does not fit the device-memory budget";
            finish_request(s, q0, Clock::now());
            s->cv_done.notify_all();
            continue;
          }
          s->cv.wait(lk);
          continue;
        }
        for (size_t k = take.size(); k-- > 0;) {
          batch.push_back(s->pending[take[k]]);
          s->pending.erase(s->pending.begin() + (std::ptrdiff_t)take[k]);
        }
        std::reverse(batch.begin(), batch.end());
        break;
      }
      sl.busy = true;
      sl.reserved = std::max(sl.reserved, need);
      s->peak = std::max(s->peak, s->reserved_total());
      if (s->active++ == 0) s->busy_from = Clock::now();
    }
    sc_status st = SC_OK;
    // a slot's page-locked parameter / column-pointer buffer, sized once for
    // the largest batch (growing it frees page-locked memory, which waits for
    // the whole device)
    if (!sl.pinned) st = sl.host_buffer(3 * align16((size_t)s->max_batch * 4) +
                                        (size_t)(s->max_batch + 1) * 8);
    if (st == SC_OK && !sl.ctx) st = create_ctx(s->device, &sl.ctx);
    if (st == SC_OK) st = run_batch(s, sl, *d, batch);
    const std::string err = st == SC_OK ? std::string() : std::string(last_error());
    {
      std::lock_guard<std::mutex> lk(s->mu);
      const Clock::time_point now = Clock::now();
      for (SrvReq* q : batch) {
        q->status = st;
        q->err = err;
        if (st != SC_OK) q->free_result();
        finish_request(s, q, now);
      }
      ++s->batches;
      s->batch_reqs += (int64_t)batch.size();
      sl.busy = false;
      if (--s->active == 0)
        s->busy_s += std::chrono::duration<double>(now - s->busy_from).count();
    }
    s->cv_done.notify_all();
    s->cv.notify_all();
  }
}

sc_status submit_at(sc_server* s, const sc_request* r, Clock::time_point t0, int64_t* ticket) {
  if (!s || !r || !ticket) return fail(SC_ERR_INVALID_ARG, "serving: null argument");
  if (r->algo != SC_REQ_OMP && r->algo != SC_REQ_LASSO)
    return fail(SC_ERR_INVALID_ARG, "serving: unknown algorithm %d", r->algo);
  if (r->n < 0 || (r->n > 0 && !r->X)) return fail(SC_ERR_INVALID_ARG, "serving: bad signals");
  if (r->precision != SC_PREC_FP32 && r->precision != SC_PREC_BF16X3)
    return fail(SC_ERR_INVALID_ARG, "unknown precision mode %d", r->precision);
  if (r->precision == SC_PREC_BF16X3 && !tc_gemm_available())
    return fail(SC_ERR_UNSUPPORTED, "BF16x3 products need the CUDA driver's tensor-map encoder");
  if (r->algo == SC_REQ_LASSO && (r->mode < 0 || r->mode > 2))
    return fail(SC_ERR_UNSUPPORTED, "lasso : mode %d not supported by the coding path", r->mode);
  SrvReq* q = new SrvReq();
  q->r = *r;
  q->t0 = t0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->dicts.find(r->dict_id);
    if (it == s->dicts.end()) {
      delete q;
      return fail(SC_ERR_INVALID_ARG, "serving: unknown dictionary id %lld", (long long)r->dict_id);
    }
    SrvDict& d = *it->second;
    const int m = d.m, K = d.K;
    if (r->algo == SC_REQ_OMP) {
      // _omp: a given L is clamped to min(m, K); without one L = min(m, K)
      q->Leff = r->L > 0 ? std::min(m, std::min(r->L, K)) : std::min(m, K);
    } else {
      // _lassoD (cpp_library/spams.h:116-130) with lambda2 = 0
      int L = r->L < 0 ? K : r->L;
      if (L > m) L = m;
      q->Leff = std::min(L, K);
    }
    q->key.dict = r->dict_id;
    q->key.algo = r->algo;
    q->key.precision = r->precision;
    q->key.refine = r->refine > 0;
    if (r->algo == SC_REQ_LASSO) {
      q->key.mode = r->mode;
      q->key.pos = r->pos != 0;
      q->key.L = q->Leff;
      q->key.path = 4 * (r->L < 0 ? K : r->L);  // length_path = 4 L before the clamp by m
    }
    q->ticket = s->next_ticket++;
    ++d.users;
    s->live[q->ticket] = q;
    *ticket = q->ticket;
    if (q->r.n == 0 || q->Leff <= 0) {
      // nothing to code: an empty K x n result at once
      q->colptr = (int64_t*)calloc((size_t)q->r.n + 1, sizeof(int64_t));
      q->rows = (int32_t*)malloc(sizeof(int32_t));
      q->vals = (float*)malloc(sizeof(float));
      finish_request(s, q, Clock::now());
      s->cv_done.notify_all();
      return SC_OK;
    }
    s->pending.push_back(q);
  }
  s->cv.notify_all();
  return SC_OK;
}

}  // namespace

extern "C" {

sc_status sc_server_create(int device, int64_t hbm_budget_bytes, int slots,
                           int64_t max_batch_signals, sc_server** out) {
  if (!out) return fail(SC_ERR_INVALID_ARG, "serving: null output");
  *out = nullptr;
  if (slots < 1 || slots > 16) return fail(SC_ERR_INVALID_ARG, "serving: slots must be 1..16");
  if (hbm_budget_bytes <= 0 || max_batch_signals <= 0)
    return fail(SC_ERR_INVALID_ARG, "serving: budget and batch size must be positive");
  DeviceCtx* admin = nullptr;
  SC_TRY(create_ctx(device, &admin));
  sc_server* s = new sc_server();
  s->device = device;
  s->budget = (size_t)hbm_budget_bytes;
  s->max_batch = max_batch_signals;
  s->admin = admin;
  for (int i = 0; i < slots; ++i) s->slots.emplace_back(new Slot());
  for (size_t i = 0; i < s->slots.size(); ++i) s->slots[i]->th = std::thread(slot_loop, s, i);
  *out = s;
  return SC_OK;
}

sc_status sc_server_destroy(sc_server* s) {
  if (!s) return SC_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;  // slots drain the queue first
  }
  s->cv.notify_all();
  for (auto& sl : s->slots)
    if (sl->th.joinable()) sl->th.join();
  cudaSetDevice(s->device);
  for (auto& sl : s->slots) {
    destroy_ctx(sl->ctx);
    for (Buf* b : {&sl->X, &sl->vecs, &sl->ocol, &sl->orows, &sl->ovals}) b->release();
    if (sl->pinned) cudaFreeHost(sl->pinned);
  }
  for (auto& kv : s->live) {
    kv.second->free_result();
    delete kv.second;
  }
  for (auto& kv : s->dicts)
    for (Buf* b : {&kv.second->D, &kv.second->Gomp, &kv.second->Glasso, &kv.second->split,
                   &kv.second->GompTc, &kv.second->GlassoTc, &kv.second->tcerr})
      b->release();
  destroy_ctx(s->admin);
  trim_pool(s->device);  // the slots' pool blocks (grown by add_dictionary) go back
  delete s;
  return SC_OK;
}

sc_status sc_server_add_dictionary_f32(sc_server* s, int64_t dict_id, const float* D, int m,
                                       int K) {
  if (!s || !D || m <= 0 || K <= 0) return fail(SC_ERR_INVALID_ARG, "serving: bad dictionary");
  SC_TRY(check_atoms(K));
  std::unique_ptr<SrvDict> d(new SrvDict());
  d->id = dict_id;
  d->m = m;
  d->K = K;
  d->Kp = pad_atoms(K);
  d->mp = tc_pad_m(m);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->dicts.count(dict_id))
      return fail(SC_ERR_INVALID_ARG, "serving: dictionary id %lld exists", (long long)dict_id);
  }
  const size_t gbytes = (size_t)d->Kp * d->Kp * 4;
  const bool tcd = tc_gemm_available();
  d->bytes = (size_t)m * K * 4 + (tcd ? 4 : 2) * gbytes + (size_t)d->mp * K * (tcd ? 6 : 4);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->reserved_total() + d->bytes > s->budget)
      return fail(SC_ERR_OUT_OF_MEMORY, "serving: dictionary does not fit the device-memory budget");
  }
  SC_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = s->admin->stream;
  SC_TRY(d->D.reserve((size_t)m * K * 4));
  SC_TRY(d->Gomp.reserve(gbytes));
  SC_TRY(d->Glasso.reserve(gbytes));
  SC_TRY(d->split.reserve((size_t)d->mp * K * (tcd ? 6 : 4)));  // hi, lo (, lo3 for the Grams)
  SC_CUDA(cudaMemcpyAsync(d->D.ptr, D, (size_t)m * K * 4, cudaMemcpyHostToDevice, st));
  const float* dD = reinterpret_cast<const float*>(d->D.ptr);
  SC_CUDA(launch_gram<float>(dD, m, K, d->Kp, 0.f, reinterpret_cast<float*>(d->Gomp.ptr), st));
  SC_CUDA(launch_gram<float>(dD, m, K, d->Kp, 1e-10f, reinterpret_cast<float*>(d->Glasso.ptr), st));
  if (tcd) {
    SC_TRY(d->GompTc.reserve(gbytes));
    SC_TRY(d->GlassoTc.reserve(gbytes));
    SC_TRY(d->tcerr.reserve(256));
    int* err = reinterpret_cast<int*>(d->tcerr.ptr);
    SC_CUDA(cudaMemsetAsync(err, 0, 4, st));
    char* sp = static_cast<char*>(d->split.ptr);
    char* lo = sp + (size_t)d->mp * K * 2;
    char* lo3 = lo + (size_t)d->mp * K * 2;
    SC_CUDA(launch_bf16_split(dD, m, m, K, d->mp, sp, lo, st, lo3));
    SC_CUDA(launch_gram_tc(sp, lo, lo3, dD, m, d->mp, K, d->Kp, 0.f,
                           reinterpret_cast<float*>(d->GompTc.ptr), err, st));
    SC_CUDA(launch_gram_tc(sp, lo, lo3, dD, m, d->mp, K, d->Kp, 1e-10f,
                           reinterpret_cast<float*>(d->GlassoTc.ptr), err, st));
    int herr = 0;
    SC_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
    SC_CUDA(cudaStreamSynchronize(st));
    if (herr) return fail(SC_ERR_TIMEOUT, "serving: a bounded tensor-core pipeline wait gave up");
  }
  SC_CUDA(cudaStreamSynchronize(st));
  size_t warm = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->dict_bytes += d->bytes;
    s->peak = std::max(s->peak, s->reserved_total());
    s->dicts[dict_id] = std::move(d);
    // the slots' workspaces come from the stream-ordered pool (AllocStream):
    // grow it now, before any request, to what every slot needs for the
    // largest batch on the largest dictionary, within the budget (growing
    // the pool by gigabytes mid-stream stalled every slot for up to a second)
    size_t need = 0;
    for (auto& kv : s->dicts) {
      const SrvDict& e = *kv.second;
      need = std::max(need, batch_bytes(e.m, e.Kp, e.mp, std::min(e.m, e.K), s->max_batch, tcd) +
                                ((size_t)256 << 20));
    }
    const size_t target = pool_target(need, s->slots.size(), s->budget, s->dict_bytes);
    if (target > s->pool_warm) {
      warm = target - s->pool_warm;
      s->pool_warm = target;
    }
  }
  if (warm > 0) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, warm, st) == cudaSuccess) {
      cudaFreeAsync(p, st);
      cudaStreamSynchronize(st);
    }
    cudaGetLastError();  // an unwarmed pool only costs time later
  }
  return SC_OK;
}

sc_status sc_server_remove_dictionary(sc_server* s, int64_t dict_id) {
  if (!s) return fail(SC_ERR_INVALID_ARG, "serving: null server");
  std::unique_ptr<SrvDict> d;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->dicts.find(dict_id);
    if (it == s->dicts.end())
      return fail(SC_ERR_INVALID_ARG, "serving: unknown dictionary id %lld", (long long)dict_id);
    if (it->second->users > 0)
      return fail(SC_ERR_INVALID_ARG, "serving: dictionary %lld has requests in flight",
                  (long long)dict_id);
    d = std::move(it->second);
    s->dicts.erase(it);
    s->dict_bytes -= d->bytes;
  }
  cudaSetDevice(s->device);
  for (Buf* b : {&d->D, &d->Gomp, &d->Glasso, &d->split, &d->GompTc, &d->GlassoTc, &d->tcerr})
    b->release();
  return SC_OK;
}

sc_status sc_server_submit(sc_server* s, const sc_request* r, int64_t* ticket) {
  return submit_at(s, r, Clock::now(), ticket);
}

sc_status sc_server_wait(sc_server* s, int64_t ticket, double timeout_s, sc_csc_f32* out,
                         double* latency_ms) {
  if (!s || !out) return fail(SC_ERR_INVALID_ARG, "serving: null argument");
  memset(out, 0, sizeof(*out));
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(ticket);
  if (it == s->live.end())
    return fail(SC_ERR_INVALID_ARG, "serving: unknown ticket %lld (already collected, or discarded)",
                (long long)ticket);
  SrvReq* q = it->second;
  if (q->r.flags & SC_REQ_DISCARD)
    return fail(SC_ERR_INVALID_ARG, "serving: request %lld discards its result", (long long)ticket);
  const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                        std::chrono::duration<double>(std::max(0.0, timeout_s)));
  while (!q->done) {
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && !q->done)
      return fail(SC_ERR_TIMEOUT, "serving: request %lld not finished within %.3f s",
                  (long long)ticket, timeout_s);
  }
  s->live.erase(it);
  std::unique_ptr<SrvReq> hold(q);
  if (latency_ms) *latency_ms = q->lat_ms;
  if (q->status != SC_OK) return fail(q->status, "%s", q->err.c_str());
  auto dd = s->dicts.find(q->r.dict_id);
  out->m = dd != s->dicts.end() ? dd->second->K : 0;
  out->n = q->r.n;
  out->nnz = q->nnz;
  out->colptr = q->colptr;
  out->rows = q->rows;
  out->vals = q->vals;
  q->colptr = nullptr;
  q->rows = nullptr;
  q->vals = nullptr;
  return SC_OK;
}

sc_status sc_server_replay(sc_server* s, const sc_request* reqs, const double* arrival_s,
                           int64_t count) {
  if (!s || (count > 0 && (!reqs || !arrival_s)))
    return fail(SC_ERR_INVALID_ARG, "serving: null argument");
  const Clock::time_point start = Clock::now() + std::chrono::milliseconds(2);
  int64_t first = -1, last = -1;
  for (int64_t i = 0; i < count; ++i) {
    const Clock::time_point at =
        start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
    std::this_thread::sleep_until(at - std::chrono::microseconds(200));
    while (Clock::now() < at) {
    }
    sc_request r = reqs[i];
    r.flags |= SC_REQ_DISCARD;
    int64_t t = 0;
    SC_TRY(submit_at(s, &r, at, &t));  // latency counts from the scheduled arrival
    if (first < 0) first = t;
    last = t;
  }
  if (first < 0) return SC_OK;
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool any = false;
    for (auto& kv : s->live)
      if (kv.first >= first && kv.first <= last) { any = true; break; }
    if (!any) break;
    s->cv_done.wait_for(lk, std::chrono::milliseconds(50));
  }
  return SC_OK;
}

sc_status sc_server_stats_get(sc_server* s, int reset, sc_server_stats* out) {
  if (!s || !out) return fail(SC_ERR_INVALID_ARG, "serving: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->completed = s->completed;
  out->signals = s->signals;
  out->batches = s->batches;
  out->rejected = s->rejected;
  snprintf(out->last_error, sizeof(out->last_error), "%s", s->last_err.c_str());
  out->lat_p50_ms = percentile(s->lat, 50);
  out->lat_p99_ms = percentile(s->lat, 99);
  double sum = 0, mx = 0;
  for (double v : s->lat) {
    sum += v;
    mx = std::max(mx, v);
  }
  out->lat_mean_ms = s->lat.empty() ? 0 : sum / (double)s->lat.size();
  out->lat_max_ms = mx;
  double busy = s->busy_s;
  if (s->active > 0) busy += std::chrono::duration<double>(Clock::now() - s->busy_from).count();
  out->busy_s = busy;
  out->peak_device_bytes = (int64_t)s->peak;
  out->mean_batch_requests = s->batches ? (double)s->batch_reqs / (double)s->batches : 0;
  out->pending = (int64_t)s->pending.size();
  if (reset) {
    s->lat.clear();
    s->completed = s->signals = s->batches = s->batch_reqs = s->rejected = 0;
    s->last_err.clear();
    s->busy_s = 0;
    if (s->active > 0) s->busy_from = Clock::now();
    s->peak = s->reserved_total();
  }
  return SC_OK;
}

}  // extern "C"
