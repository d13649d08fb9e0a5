// Request queue of linear solves behind the C ABI (no counterpart in the
// reference, which solves one model per call of StaticSolver.solve,
// gfem/solvers.py:481-605): a host that is not Python submits right-hand sides
// against resident solver handles and collects the solutions later.
//
// `workers` host threads each own a CUDA stream on the queue's device and
// grow-only device vectors.  A worker takes the oldest pending request whose
// solver is idle (a solver handle serves one request at a time: its workspace and
// captured graphs are per handle), copies the right-hand side to the device,
// runs exfem_solver_mixed on its stream (FP32 matrix-free PCG inside FP64
// refinement, the solver's mixed mode), and copies the solution back into the
// request.  Requests of different solvers run concurrently on the workers'
// streams.  Pending requests can be withdrawn; finished ones stay until their
// result is collected.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "solver.h"

namespace exfem {

struct Request {
  int64_t id = 0;
  exfem_solver_s* solver = nullptr;
  std::vector<double> rhs, x;
  double tol = 1e-8;
  int state = EXFEM_REQ_PENDING;
  int status = EXFEM_OK;
  int iters = 0, passes = 0;
  double relres = 0.0;
  std::string error;
};

}  // namespace exfem

struct exfem_queue_s {
  int device = 0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<exfem::Request*> pending;
  std::map<int64_t, std::unique_ptr<exfem::Request>> all;   // every request not yet collected
  std::map<exfem_solver_s*, bool> busy;
  int64_t next_id = 1;
  bool stop = false;
  std::vector<std::thread> threads;
  void worker();
};

void exfem_queue_s::worker() {
  using namespace exfem;
  cudaSetDevice(device);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  DevBuf<double> b, x;
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lock(mu);
      for (;;) {
        if (stop) {
          if (st) cudaStreamDestroy(st);
          return;
        }
        for (auto it = pending.begin(); it != pending.end(); ++it)
          if (!busy[(*it)->solver]) {
            r = *it;
            pending.erase(it);
            break;
          }
        if (r) break;
        cv.wait(lock);
      }
      r->state = EXFEM_REQ_RUNNING;
      busy[r->solver] = true;
    }
    const int64_t n = r->solver->n;
    int s = EXFEM_OK;
    if ((size_t)n > b.n && ((s = b.alloc(n)) || (s = x.alloc(n)))) {
    } else if (cudaMemcpyAsync(b.p, r->rhs.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      s = EXFEM_ERR_CUDA;
      set_error("request %lld: copy of the right-hand side failed", (long long)r->id);
    } else {
      s = exfem_solver_mixed(r->solver, b.p, x.p, r->tol, 2e-5, 12, 20000, &r->iters, &r->passes, &r->relres, st);
      if (s >= 0) {
        r->x.resize(n);
        if (cudaMemcpyAsync(r->x.data(), x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
          s = EXFEM_ERR_CUDA;
          set_error("request %lld: copy of the solution failed", (long long)r->id);
        }
      }
    }
    const std::string msg = s < 0 ? std::string(exfem_last_error()) : std::string();
    {
      std::lock_guard<std::mutex> lock(mu);
      r->status = s;
      r->error = msg;
      r->state = s < 0 ? EXFEM_REQ_FAILED : EXFEM_REQ_DONE;
      r->rhs.clear();
      r->rhs.shrink_to_fit();
      busy[r->solver] = false;
    }
    cv.notify_all();
  }
}

extern "C" {

int exfem_queue_create(int workers, exfem_queue* out) try {
  EX_ARG(out, "out is NULL");
  *out = nullptr;
  EX_ARG(workers >= 1 && workers <= 64, "workers must lie in 1..64, got %d", workers);
  auto q = std::make_unique<exfem_queue_s>();
  EX_CUDA(cudaGetDevice(&q->device));
  for (int i = 0; i < workers; ++i) q->threads.emplace_back([p = q.get()] { p->worker(); });
  *out = q.release();
  return EXFEM_OK;
} catch (...) {
  return ::exfem::host_exception();
}

int exfem_queue_destroy(exfem_queue q) {
  if (!q) return EXFEM_OK;
  {
    std::lock_guard<std::mutex> lock(q->mu);
    for (auto* r : q->pending) r->state = EXFEM_REQ_CANCELLED;
    q->pending.clear();
    q->stop = true;
  }
  q->cv.notify_all();
  for (auto& t : q->threads) t.join();      // a running request finishes first
  delete q;
  return EXFEM_OK;
}

int exfem_queue_submit(exfem_queue q, exfem_solver s, const double* rhs_host, double tol, int64_t* id) try {
  EX_ARG(q && s && rhs_host && id, "NULL argument");
  EX_ARG(s->op == EXFEM_OP_MF_F32, "queued solves run the mixed solver: the handle needs EXFEM_OP_MF_F32");
  EX_ARG(tol > 0, "tolerance must be positive, got %g", tol);
  auto r = std::make_unique<exfem::Request>();
  r->solver = s;
  r->rhs.assign(rhs_host, rhs_host + s->n);
  r->tol = tol;
  {
    std::lock_guard<std::mutex> lock(q->mu);
    EX_ARG(!q->stop, "queue is closing");
    r->id = q->next_id++;
    *id = r->id;
    q->pending.push_back(r.get());
    q->all[r->id] = std::move(r);
  }
  q->cv.notify_all();
  return EXFEM_OK;
} catch (...) {
  return ::exfem::host_exception();
}

int exfem_queue_poll(exfem_queue q, int64_t id, int* state, int* iters, double* relres) {
  EX_ARG(q && state, "NULL argument");
  std::lock_guard<std::mutex> lock(q->mu);
  auto it = q->all.find(id);
  EX_ARG(it != q->all.end(), "no request %lld in the queue (unknown or already collected)", (long long)id);
  *state = it->second->state;
  if (iters) *iters = it->second->iters;
  if (relres) *relres = it->second->relres;
  return EXFEM_OK;
}

int exfem_queue_wait(exfem_queue q, int64_t id, double timeout_s, int* state) {
  EX_ARG(q && state, "NULL argument");
  std::unique_lock<std::mutex> lock(q->mu);
  auto it = q->all.find(id);
  EX_ARG(it != q->all.end(), "no request %lld in the queue (unknown or already collected)", (long long)id);
  exfem::Request* r = it->second.get();
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (r->state == EXFEM_REQ_PENDING || r->state == EXFEM_REQ_RUNNING)
    if (q->cv.wait_until(lock, until) == std::cv_status::timeout) break;
  *state = r->state;
  return EXFEM_OK;
}

int exfem_queue_result(exfem_queue q, int64_t id, double* x_host, int* iters, int* passes, double* relres) {
  EX_ARG(q, "queue is NULL");
  std::unique_ptr<exfem::Request> r;
  {
    std::lock_guard<std::mutex> lock(q->mu);
    auto it = q->all.find(id);
    EX_ARG(it != q->all.end(), "no request %lld in the queue (unknown or already collected)", (long long)id);
    const int state = it->second->state;
    EX_ARG(state == EXFEM_REQ_DONE || state == EXFEM_REQ_FAILED || state == EXFEM_REQ_CANCELLED,
           "request %lld has not finished (state %d)", (long long)id, state);
    r = std::move(it->second);
    q->all.erase(it);
  }
  if (r->state == EXFEM_REQ_CANCELLED) {
    exfem::set_error("request %lld was withdrawn", (long long)id);
    return EXFEM_ERR_ARG;
  }
  if (r->state == EXFEM_REQ_FAILED) {
    exfem::set_error("request %lld failed: %s", (long long)id, r->error.c_str());
    return r->status;
  }
  if (x_host) std::copy(r->x.begin(), r->x.end(), x_host);
  if (iters) *iters = r->iters;
  if (passes) *passes = r->passes;
  if (relres) *relres = r->relres;
  return r->status;
}

int exfem_queue_cancel(exfem_queue q, int64_t id, int* withdrawn) {
  EX_ARG(q && withdrawn, "NULL argument");
  std::lock_guard<std::mutex> lock(q->mu);
  auto it = q->all.find(id);
  EX_ARG(it != q->all.end(), "no request %lld in the queue (unknown or already collected)", (long long)id);
  *withdrawn = 0;
  exfem::Request* r = it->second.get();
  if (r->state != EXFEM_REQ_PENDING) return EXFEM_OK;
  for (auto p = q->pending.begin(); p != q->pending.end(); ++p)
    if (*p == r) {
      q->pending.erase(p);
      break;
    }
  r->state = EXFEM_REQ_CANCELLED;
  *withdrawn = 1;
  q->cv.notify_all();
  return EXFEM_OK;
}

}  // extern "C"
