// Request server: continuous batching of boundary-value solves on one GPU.
//
// Requests (a bemgpu_problem: mesh, media, lattice, frequency, incidence) are
// queued on submit and admitted to solver slots as slots and device memory
// free up.  Each slot owns a context (its own CUDA streams and solver
// scratch) and a host worker thread, so the assemblies and solves of
// admitted requests overlap on the device.  A slot keeps its last problem's
// matrices and factors; a request whose reuse key (mesh, media, lattice,
// frequency, in-plane Bloch wave vector, precision) matches an idle slot's is
// routed there and only its right-hand side is solved; a request on the same
// body, media and frequency as a slot's resident problem (another Bloch wave
// vector) is preferred there, and the context keeps the free-space domains'
// matrices and dpv factors (bemgpu_interior_reuses).  Admission keeps the
// sum of the resident problems' device bytes (N^2 16 B per matrix plus
// workspace, see problem_bytes) within the budget; idle slots' problems are
// evicted, least recently used first, to make room.  Later requests that fit
// may pass a request that does not (backfilling), until the waiting request
// is older than BACKFILL_MS.  A request whose reuse key is being solved in a
// busy slot, or by an earlier queued request, waits for those factors without
// a time limit, letting later requests pass.
//
// The reference has no server: each request is one solve_bieq_aqd2 +
// force_FN_aqd2 (bem3_aw_qd2_solve_bieq.c:3, bem3_aw_qd2_force.c:4).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include "../../include/bemgpu.h"

#define BACKFILL_MS 2000.0

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// a deep copy of a bemgpu_problem (the caller may free its arrays after submit)
struct owned_problem {
  std::vector<double> cr, cw, ren, wen, k0, k2, rho0, c0, Pi, dPi, p_inc, v_inc, xl, wl, xh, wh;
  std::vector<int> npe, eni, md, sd, dom_ne, sid;
  std::vector<unsigned char> plane;
  bemgpu_problem p;

  template <class T>
  static void copy(std::vector<T> &v, const T *src, size_t n) { v.assign(src, src + n); }

  explicit owned_problem(const bemgpu_problem *s) {
    const size_t Ne = s->Ne, nd = s->MN + 1;
    size_t tot = 0;
    for (size_t d = 0; d < nd; ++d) tot += s->dom_ne[d];
    copy(cr, s->cr, Ne * 12); copy(cw, s->cw, Ne * 9); copy(ren, s->ren, Ne * 12); copy(wen, s->wen, Ne * 12);
    copy(npe, s->npe, Ne); copy(eni, s->eni, Ne * 4); copy(md, s->md, Ne); copy(sd, s->sd, Ne);
    copy(dom_ne, s->dom_ne, nd); copy(sid, s->sid, tot);
    copy(k0, s->k0, nd); copy(k2, s->k2, 2 * nd); copy(rho0, s->rho0, nd); copy(c0, s->c0, nd);
    copy(Pi, s->Pi, Ne * 8); copy(dPi, s->dPi, Ne * 8); copy(p_inc, s->p_inc, Ne * 8); copy(v_inc, s->v_inc, Ne * 24);
    copy(xl, s->xl, 12); copy(wl, s->wl, 12); copy(xh, s->xh, 64); copy(wh, s->wh, 64);
    copy(plane, s->plane, Ne);
    p = *s;
    p.cr = cr.data(); p.cw = cw.data(); p.ren = ren.data(); p.wen = wen.data();
    p.npe = npe.data(); p.eni = eni.data(); p.md = md.data(); p.sd = sd.data();
    p.dom_ne = dom_ne.data(); p.sid = sid.data(); p.k0 = k0.data(); p.k2 = k2.data();
    p.rho0 = rho0.data(); p.c0 = c0.data(); p.Pi = Pi.data(); p.dPi = dPi.data();
    p.p_inc = p_inc.data(); p.v_inc = v_inc.data(); p.xl = xl.data(); p.wl = wl.data();
    p.xh = xh.data(); p.wh = wh.data(); p.plane = plane.data();
  }
};

// device bytes a resident problem holds: global matrix n^2 16 B, per domain
// G, H, dpv factors 3 N_d^2 16 B (+ dG, dH 4 N_d^2 16 B for interior domains
// when they are kept, else one 512 MiB block of recomputed rows), FP32 factors
// in mixed precision, and element tables / scratch
size_t problem_bytes(const bemgpu_problem *p, int precision, bool keep_dgh) {
  const size_t n = 2 * (size_t)p->NN;
  size_t b = n * n * 16, f32 = n * n * 8;
  for (int d = 0; d <= p->MN; ++d) {
    const size_t N = 4 * (size_t)p->dom_ne[d];
    // matrices, pair flags (and the periodic domain's 4-byte pair lists), near-singular tables
    b += 3 * N * N * 16 + (d > 0 && keep_dgh ? 4 * N * N * 16 : 0) + N * (size_t)p->dom_ne[d] * (d == 0 ? 5 : 1) +
         N * 256 * 28;
    f32 += N * N * 8;
  }
  if (precision) b += f32;
  if (!keep_dgh && p->MN >= 1) b += (size_t)512 << 20;
  return b + (size_t)p->Ne * 512 + (64u << 20);  // tables, workspace of the solvers
}

// FNV-1a over what the free-space (interior) domains' matrices depend on (the
// element tables, domain lists and interior wave numbers; the context itself
// compares the data exactly before it keeps anything)
unsigned long long interior_key(const bemgpu_problem *p) {
  unsigned long long h = 1469598103934665603ull;
  auto put = [&h](const void *src, size_t bytes) {
    const unsigned char *b = (const unsigned char *)src;
    for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
  };
  const size_t ne = p->Ne;
  size_t tot = 0;
  for (int d = 0; d <= p->MN; ++d) tot += p->dom_ne[d];
  put(&p->Ne, sizeof(int)); put(&p->MN, sizeof(int));
  put(p->dom_ne, sizeof(int) * (p->MN + 1)); put(p->sid, sizeof(int) * tot);
  put(p->cr, sizeof(double) * 12 * ne); put(p->cw, sizeof(double) * 9 * ne);
  put(p->ren, sizeof(double) * 12 * ne); put(p->wen, sizeof(double) * 12 * ne);
  put(p->npe, sizeof(int) * ne); put(p->plane, ne);
  put(p->k0 + 1, sizeof(double) * p->MN);
  return h;
}

struct request {
  long long id;
  owned_problem prob;
  unsigned long long key, ikey;
  int precision, force_type;
  bool keep_dgh = true;  // interior derivative rows kept (false: recomputed in blocks)
  double rc[3];
  size_t bytes;
  double t_submit, t_start = 0;
  request(const bemgpu_problem *p, unsigned long long k, int prec, int ft, const double *r, long long i)
      : id(i), prob(p), key(k), ikey(interior_key(p)), precision(prec), force_type(ft),
        bytes(problem_bytes(p, prec, true)), t_submit(now_ms()) {
    for (int j = 0; j < 3; ++j) rc[j] = r ? r[j] : 0.0;
  }
};

struct slot {
  bemgpu_ctx *ctx = nullptr;
  std::thread th;
  request *cur = nullptr;        // assigned request (owned by the slot while running)
  unsigned long long key = 0;    // reuse key of the resident problem
  unsigned long long ikey = 0;   // interior key of the resident problem
  int precision = -1;
  bool keep_dgh = true;          // the resident problem's interior derivative rows are kept
  bool resident = false;         // a problem (and its factors) is loaded
  bool evict = false;            // free the resident problem before the next request
  size_t bytes = 0;              // device bytes of the resident problem
  double last_used = 0;
};

}  // namespace

struct bemgpu_server {
  int device = 0;
  size_t budget = 0, used = 0, peak = 0;
  std::vector<slot> slots;
  std::deque<request *> queue;
  std::deque<bemgpu_result> done;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  long long submitted = 0, completed = 0, reused = 0, evictions = 0, failed = 0;
};

static void dispatch_locked(bemgpu_server *s) {
  const double t = now_ms();
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    request *r = *it;
    int pick = -1;
    // 1. an idle slot holding this request's factors
    for (size_t i = 0; i < s->slots.size(); ++i) {
      slot &sl = s->slots[i];
      if (!sl.cur && sl.resident && !sl.evict && sl.key == r->key && sl.precision == r->precision) { pick = (int)i; break; }
    }
    if (pick < 0) {
      // a busy slot computes this request's matrices, or an earlier queued
      // request will: wait for those factors rather than assembling the same
      // matrices a second time, however long that takes (the factors arrive no
      // later than a second assembly started now would finish; if the other
      // request fails, this one is admitted on its own at the next dispatch)
      bool pending = false;
      for (auto &sl : s->slots)
        if (sl.cur && sl.cur->key == r->key && sl.cur->precision == r->precision) pending = true;
      for (auto jt = s->queue.begin(); jt != it && !pending; ++jt)
        if ((*jt)->key == r->key && (*jt)->precision == r->precision) pending = true;
      if (pending) { ++it; continue; }
    }
    if (pick < 0) {
      // 2. an idle slot whose resident problem can be replaced within the budget;
      //    evict idle slots (least recently used first) if that makes room
      std::vector<int> idle;
      for (size_t i = 0; i < s->slots.size(); ++i)
        if (!s->slots[i].cur) idle.push_back((int)i);
      if (!idle.empty()) {
        // replace first: a slot with this request's interior matrices, then
        // empty slots, then slots whose factors no queued request wants,
        // least recently used first
        auto same_interior = [&](const slot &x) {
          return x.resident && x.ikey == r->ikey && x.precision == r->precision;
        };
        auto wanted = [&](const slot &x) {
          if (!x.resident) return false;
          for (request *q : s->queue)
            if (q != r && q->key == x.key && q->precision == x.precision) return true;
          return false;
        };
        std::sort(idle.begin(), idle.end(), [&](int a, int b) {
          const slot &x = s->slots[a], &y = s->slots[b];
          const bool ix = same_interior(x), iy = same_interior(y);
          if (ix != iy) return ix;
          if (x.resident != y.resident) return !x.resident;
          const bool wx = wanted(x), wy = wanted(y);
          if (wx != wy) return !wx;
          return x.last_used < y.last_used;
        });
        size_t used = s->used;
        const int target = idle[0];
        used -= s->slots[target].bytes;
        std::vector<int> evict;
        for (size_t k = 1; k < idle.size() && used + r->bytes > s->budget; ++k)
          if (s->slots[idle[k]].resident) {
            used -= s->slots[idle[k]].bytes;
            evict.push_back(idle[k]);
          }
        if (used + r->bytes <= s->budget) {
          pick = target;
          for (int e : evict) {
            slot &sl = s->slots[e];
            sl.evict = true;  // the worker frees it; its bytes leave the budget now
            s->used -= sl.bytes;
            sl.bytes = 0;
            sl.resident = false;
            ++s->evictions;
          }
          s->used -= s->slots[target].bytes;
          s->slots[target].bytes = 0;
        }
      }
    }
    if (pick >= 0) {
      slot &sl = s->slots[pick];
      if (!(sl.resident && sl.key == r->key && sl.precision == r->precision && sl.bytes)) {
        sl.bytes = r->bytes;
        s->used += r->bytes;
        if (s->used > s->peak) s->peak = s->used;
      }
      r->t_start = t;
      sl.cur = r;
      it = s->queue.erase(it);
      continue;
    }
    // the head waits too long: no backfilling past it
    if (t - r->t_submit > BACKFILL_MS) break;
    ++it;
  }
  s->cv_work.notify_all();
}

static void worker(bemgpu_server *s, int idx) {
  cudaSetDevice(s->device);
  for (;;) {
    request *r = nullptr;
    bool evict = false;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || s->slots[idx].cur != nullptr || s->slots[idx].evict; });
      slot &sl = s->slots[idx];
      if (sl.evict) { evict = true; sl.evict = false; }
      r = sl.cur;
      if (!r && s->stop) return;
    }
    slot &sl = s->slots[idx];
    if (evict) bemgpu_unload(sl.ctx);
    if (!r) continue;
    bemgpu_result res;
    memset(&res, 0, sizeof(res));
    res.id = r->id;
    bool reuse = sl.resident && sl.key == r->key && sl.precision == r->precision;
    int rc = 0;
    if (reuse) {
      const bemgpu_problem &p = r->prob.p;
      rc = bemgpu_set_incident(sl.ctx, p.Pi, p.dPi, p.p_inc, p.v_inc, p.pw);
      if (!rc) rc = bemgpu_solve_rhs(sl.ctx);
      if (rc == -2) reuse = false;  // factors no longer held: full solve below
    }
    if (!reuse) {
      // the slot's device memory is what admission counted for this problem:
      // give back the previous problem's buffers instead of reusing them,
      // unless the problem is on the same body at the same frequency, whose
      // buffers have this problem's sizes and whose interior matrices and
      // factors the context keeps
      const bool same_interior =
          sl.resident && sl.ikey == r->ikey && sl.precision == r->precision && sl.keep_dgh == r->keep_dgh;
      sl.resident = false;
      rc = same_interior ? 0 : bemgpu_unload(sl.ctx);
      if (!rc && !same_interior) rc = bemgpu_set_precision(sl.ctx, r->precision);
      if (!rc && !same_interior) rc = bemgpu_set_interior_derivatives(sl.ctx, r->keep_dgh ? 1 : 0, 0);
      if (!rc) rc = bemgpu_load(sl.ctx, &r->prob.p);
      if (!rc) rc = bemgpu_run(sl.ctx);
    }
    if (!rc) rc = bemgpu_force(sl.ctx, r->force_type, r->rc, res.F, res.N);
    if (!rc) rc = bemgpu_sync(sl.ctx);
    if (!rc && bemgpu_status(sl.ctx)) rc = -5;
    const double t_end = now_ms();
    res.status = rc;
    res.reused = reuse ? 1 : 0;
    res.precision = r->precision;
    res.queue_ms = r->t_start - r->t_submit;
    res.service_ms = t_end - r->t_start;
    if (rc) snprintf(res.error, sizeof(res.error), "%s", bemgpu_error(sl.ctx));
    {
      std::lock_guard<std::mutex> lk(s->mu);
      sl.cur = nullptr;
      sl.last_used = t_end;
      if (rc) {
        // a failed request leaves nothing reusable behind
        bemgpu_unload(sl.ctx);
        s->used -= sl.bytes;
        sl.bytes = 0;
        sl.resident = false;
        ++s->failed;
      } else {
        sl.resident = true;
        sl.key = r->key;
        sl.ikey = r->ikey;
        sl.precision = r->precision;
        sl.keep_dgh = r->keep_dgh;
        if (reuse) ++s->reused;
      }
      ++s->completed;
      s->done.push_back(res);
      delete r;
      dispatch_locked(s);
    }
    s->cv_done.notify_all();
  }
}

extern "C" int bemgpu_server_create(int device, size_t hbm_budget, int nslots, bemgpu_server **out) {
  *out = nullptr;
  if (nslots < 1 || nslots > 64) return -2;
  bemgpu_server *s = new bemgpu_server();
  s->device = device;
  s->budget = hbm_budget;
  s->slots.resize(nslots);
  for (int i = 0; i < nslots; ++i)
    if (bemgpu_create(device, nullptr, &s->slots[i].ctx) != 0) {
      for (int j = 0; j < i; ++j) bemgpu_destroy(s->slots[j].ctx);
      delete s;
      return -1;
    }
  for (int i = 0; i < nslots; ++i) s->slots[i].th = std::thread(worker, s, i);
  *out = s;
  return 0;
}

extern "C" int bemgpu_server_submit(bemgpu_server *s, const bemgpu_problem *p, unsigned long long reuse_key,
                                    int precision, int force_type, const double *rc, long long id) {
  request *r = new request(p, reuse_key, precision, force_type, rc, id);
  std::lock_guard<std::mutex> lk(s->mu);
  if (r->bytes > s->budget) {
    // too large as asked: first recompute the interior derivative rows in
    // blocks instead of keeping them, then give up the FP32 factors (FP64
    // with the rows kept, then recomputed)
    const int prec = r->precision;
    const struct { int prec; bool keep; } tries[3] = {{prec, false}, {0, true}, {0, false}};
    for (const auto &tr : tries) {
      r->precision = tr.prec;
      r->keep_dgh = tr.keep;
      r->bytes = problem_bytes(p, tr.prec, tr.keep);
      if (r->bytes <= s->budget) break;
    }
  }
  if (r->bytes > s->budget) { delete r; return -2; }  // can never be admitted
  s->queue.push_back(r);
  ++s->submitted;
  dispatch_locked(s);
  return 0;
}

extern "C" int bemgpu_server_poll(bemgpu_server *s, bemgpu_result *out, int max, int timeout_ms) {
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && timeout_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty(); });
  int k = 0;
  while (k < max && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  return k;
}

extern "C" int bemgpu_server_stats(bemgpu_server *s, double *out8) {
  std::lock_guard<std::mutex> lk(s->mu);
  int running = 0;
  for (auto &sl : s->slots) running += sl.cur != nullptr;
  out8[0] = (double)s->submitted;
  out8[1] = (double)s->completed;
  out8[2] = (double)s->reused;
  out8[3] = (double)running;
  out8[4] = (double)s->queue.size();
  out8[5] = (double)s->used;
  out8[6] = (double)s->peak;
  out8[7] = (double)s->evictions;
  return 0;
}

extern "C" void bemgpu_server_destroy(bemgpu_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (request *r : s->queue) delete r;
    s->queue.clear();
  }
  s->cv_work.notify_all();
  for (auto &sl : s->slots)
    if (sl.th.joinable()) sl.th.join();
  for (auto &sl : s->slots) bemgpu_destroy(sl.ctx);
  delete s;
}
