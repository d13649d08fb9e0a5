// extern "C" entry points of libexfem_b200 (declared in include/exfem_b200.h).
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <new>
#include <stdexcept>

#include "sa.h"
#include "solver.h"

namespace exfem {

static thread_local std::string g_err;
// elements per matrix-free tile for blocks created from now on: C3D8, C3D10
static int g_tile[2] = {128, 256};

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

int cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  set_error("%s failed (%s:%d): %s", what, file, line, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? EXFEM_ERR_OOM : EXFEM_ERR_CUDA;
}

int host_exception() {
  try {
    throw;
  } catch (const std::bad_alloc&) {
    set_error("host memory exhausted");
    return EXFEM_ERR_OOM;
  } catch (const std::length_error&) {
    set_error("size too large for a host array");
    return EXFEM_ERR_ARG;
  } catch (const std::exception& e) {
    set_error("host error: %s", e.what());
    return EXFEM_ERR_UNSUPPORTED;
  } catch (...) {
    set_error("unknown host error");
    return EXFEM_ERR_UNSUPPORTED;
  }
}

int host_gather_plan(int64_t nn, int64_t ne, int nnode, const int32_t* conn, std::vector<int32_t>* plan, int& vmax);
int host_colouring(int64_t nn, int64_t ne, int nnode, const int32_t* conn, std::vector<int32_t>& colour, int& ncolour);
int host_standard_aggregation(int64_t n, const int64_t* ptr, const int32_t* idx, int32_t* agg, int64_t& nagg);
int host_tile_order(int64_t nn, int64_t ne, int nnode, int ncorner, const double* X, const int32_t* conn,
                    std::vector<int32_t>& order);
int host_tile_pairs(int64_t ne, const int32_t* conn, std::vector<int32_t>& order, std::vector<int32_t>& conn_tile);
int host_face_once(int64_t nface, const int64_t* keys, uint8_t* once);
int host_tile_maps(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int tile, std::vector<int32_t>& ptr,
                   std::vector<int32_t>& nodes, std::vector<uint16_t>& nend, std::vector<uint16_t>& perm, int& maxu);
int solver_pcg(exfem_solver_s* S, const double* b, double* x, double tol, int maxiter, int* iters, double* relres, cudaStream_t st);
int newton_increment(exfem_solver_s* S, const double* u, const double* const* s_old, const double* fext,
                     const double* start, double rtol, int max_iter, int line_search, double cg_tol, int cg_maxiter,
                     double* qref, double* u_out, double* const* s_out, int* corrections, int* converged,
                     double* hist, int* lin_stats, cudaStream_t st);
int solver_mixed_graph(exfem_solver_s* S, const double* b, double* x, double tol, double delta, int max_updates,
                       int maxiter, int* iters, int* updates, double* relres, cudaStream_t st);
int solver_mixed_ru(exfem_solver_s* S, const double* b, double* x, double tol, double delta, int max_updates,
                    int maxiter, int* iters, int* updates, double* relres, cudaStream_t st);
int solver_mixed(exfem_solver_s* S, const double* b, double* x, double tol, double inner_tol, int max_pass,
                 int maxiter, int* iters, int* passes, double* relres, cudaStream_t st);
int solver_refresh_diagonal(exfem_solver_s* S, cudaStream_t st);
int solver_alloc(exfem_solver_s* S);

// a bounded wait inside one of the block's kernels gave up (a copy or a tensor-core
// operation that did not complete): report it once and clear the flag
int block_wait_status(exfem_block_s* b, cudaStream_t s) {
  if (!b->dev_err.p) return EXFEM_OK;
  int h = 0;
  EX_CUDA(cudaMemcpyAsync(&h, b->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  EX_CUDA(cudaStreamSynchronize(s));
  if (!h) return EXFEM_OK;
  EX_CUDA(cudaMemsetAsync(b->dev_err.p, 0, sizeof(int), s));
  set_error("a bounded device wait gave up (an asynchronous copy or tensor-core operation did not complete); "
            "the results of the call are invalid");
  return EXFEM_ERR_TIMEOUT;
}

static int set_material(exfem_block_s* b, const exfem_material* m) {
  EX_ARG(m, "material is NULL");
  EX_ARG(m->kind == EXFEM_LINEAR_ELASTIC || m->kind == EXFEM_J2, "unknown material kind %d", m->kind);
  EX_ARG(m->E > 0 && m->nu > -1.0 && m->nu < 0.5, "invalid elastic constants E=%g nu=%g", m->E, m->nu);
  b->mat_in = *m;
  MatDev& d = b->mat;
  memset(&d, 0, sizeof(d));
  d.kind = m->kind;
  d.mu = m->E / (2.0 * (1.0 + m->nu));                        // gfem/materials.py:18-19
  d.lam = m->E * m->nu / ((1.0 + m->nu) * (1.0 - 2.0 * m->nu));
  d.K = d.lam + 2.0 * d.mu / 3.0;                             // gfem/materials.py:245
  d.Hk = m->Hk;
  if (m->kind == EXFEM_J2) {
    EX_ARG(m->ntab >= 2 && m->ntab <= EXFEM_MAX_TABLE, "J2 table needs 2..%d rows, got %d", EXFEM_MAX_TABLE, m->ntab);
    for (int i = 1; i < m->ntab; ++i)
      EX_ARG(m->ep_tab[i] >= m->ep_tab[i - 1], "J2 table plastic strains must be non-decreasing");
    d.ntab = m->ntab;
    for (int i = 0; i < m->ntab; ++i) {
      d.ep[i] = m->ep_tab[i];
      d.sy[i] = m->sy_tab[i];
    }
  }
  return EXFEM_OK;
}

static int init_tangent(exfem_block_s* b) {
  if (b->mat.kind != EXFEM_J2) return EXFEM_OK;
  // elastic tangent data (c1 = 1) in the tile-major layout, padding included
  const int W = b->ngp * 8;
  const size_t n = (size_t)b->ntile * b->tile * W;
  std::vector<double> t(n, 0.0);
  std::vector<float> t32(n, 0.0f);
  for (int64_t p = 0; p < b->ntile * b->tile; ++p)
    for (int g = 0; g < b->ngp; ++g) {
      t[tile_index(p, g * 8 + 6, W, b->tile)] = 1.0;
      t32[tile_index(p, g * 8 + 6, W, b->tile)] = 1.0f;
    }
  int s;
  if ((s = b->tan64.upload(t.data(), n))) return s;
  return b->tan32.upload(t32.data(), n);
}

}  // namespace exfem

using namespace exfem;

static cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

template <class T>
static int mf_apply_cb(void* ctx, const T* x, T* y, const int* skip, cudaStream_t s) {
  return launch_mf_matvec<T>((exfem_block_s*)ctx, x, y, skip, s);
}

// graphs cannot be captured on the legacy default stream: such calls run on a
// private stream ordered after and before the caller's stream with events
namespace exfem {
std::shared_mutex& capture_lock() {
  static std::shared_mutex m;
  return m;
}

int& capturing_here() {
  static thread_local int c = 0;
  return c;
}
}  // namespace exfem

struct StreamGuard {
  cudaStream_t user, work = nullptr;
  cudaEvent_t ev = nullptr;
  bool own = false;
  int init(void* s) {
    user = (cudaStream_t)s;
    if (user != nullptr && user != cudaStreamLegacy) { work = user; return EXFEM_OK; }
    EX_CUDA(cudaStreamCreateWithFlags(&work, cudaStreamNonBlocking));
    EX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    own = true;
    EX_CUDA(cudaEventRecord(ev, user));
    EX_CUDA(cudaStreamWaitEvent(work, ev, 0));
    return EXFEM_OK;
  }
  ~StreamGuard() {
    if (own) {
      cudaEventRecord(ev, work);
      cudaStreamWaitEvent(user, ev, 0);
      cudaEventDestroy(ev);
      cudaStreamDestroy(work);
    }
  }
};

// Host work behind a C entry point: a C++ exception must not cross the C ABI, so
// an allocation that fails (or a size no host array can hold) becomes a status
template <class F>
static int host_guard(F&& f) {
  try {
    return f();
  } catch (...) {
    return host_exception();
  }
}

extern "C" {

int exfem_version(void) { return 1000; }
const char* exfem_last_error(void) { return g_err.c_str(); }

int exfem_block_create(int etype, const exfem_material* mat, int64_t nn, const double* X_host, int64_t ne,
                       const int32_t* conn_host, exfem_block* out) try {
  EX_ARG(out, "out is NULL");
  *out = nullptr;
  EX_ARG(etype == EXFEM_C3D8 || etype == EXFEM_C3D10, "unknown element type %d", etype);
  EX_ARG(nn >= 0 && ne >= 0, "negative sizes");
  EX_ARG(nn == 0 || X_host, "X is NULL");
  EX_ARG(ne == 0 || conn_host, "conn is NULL");
  EX_ARG(3 * nn < (int64_t)INT32_MAX && nn < (int64_t(1) << 28), "too many nodes for int32 DOF indices");
  auto b = std::make_unique<exfem_block_s>();
  cudaGetDevice(&b->device);
  b->etype = etype;
  b->nnode = etype == EXFEM_C3D8 ? 8 : 10;
  b->ngp = etype == EXFEM_C3D8 ? 8 : 4;
  b->nd = 3 * b->nnode;
  b->ne = ne;
  b->nn = nn;
  int s;
  if ((s = set_material(b.get(), mat))) return s;
  b->nstate = mat->kind == EXFEM_J2 ? 19 : 1;
  if ((s = host_gather_plan(nn, ne, b->nnode, conn_host, &b->plan_host, b->vmax))) return s;
  std::vector<int32_t> colours;
  if ((s = host_colouring(nn, ne, b->nnode, conn_host, colours, b->ncolour))) return s;
  b->colour_host = colours;
  // elements grouped by colour, ascending element index within a colour
  b->colour_ptr.assign(b->ncolour + 1, 0);
  for (int64_t e = 0; e < ne; ++e) ++b->colour_ptr[colours[e] + 1];
  for (int c = 0; c < b->ncolour; ++c) b->colour_ptr[c + 1] += b->colour_ptr[c];
  std::vector<int32_t> elems(ne);
  {
    std::vector<int64_t> pos(b->colour_ptr.begin(), b->colour_ptr.end() - 1);
    for (int64_t e = 0; e < ne; ++e) elems[pos[colours[e]]++] = (int32_t)e;
  }
  // straight-edge check for C3D10 (mid-node at the edge midpoint)
  b->affine = 1;
  if (etype == EXFEM_C3D10) {
    static const int E[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    for (int64_t e = 0; e < ne && b->affine; ++e) {
      const int32_t* c = conn_host + e * 10;
      for (int k = 0; k < 6; ++k) {
        const double* p = X_host + 3 * (int64_t)c[E[k][0]];
        const double* q = X_host + 3 * (int64_t)c[E[k][1]];
        const double* m = X_host + 3 * (int64_t)c[4 + k];
        double L = 0.0, d = 0.0;
        for (int i = 0; i < 3; ++i) {
          L += (q[i] - p[i]) * (q[i] - p[i]);
          const double r = m[i] - 0.5 * (p[i] + q[i]);
          d += r * r;
        }
        if (d > 1e-20 * L) { b->affine = 0; break; }
      }
    }
  }
  {
    // tile order: elements by mesh component, then along a Morton curve
    b->tile = g_tile[etype == EXFEM_C3D8 ? 0 : 1];
    if ((s = host_tile_order(nn, ne, b->nnode, etype == EXFEM_C3D8 ? 8 : 4, X_host, conn_host, b->order_host)))
      return s;
    std::vector<int32_t> conn_ord((size_t)ne * b->nnode), tpos(ne);
    if (etype == EXFEM_C3D10 && b->mat.kind == EXFEM_LINEAR_ELASTIC) {
      // face-sharing pairs side by side, in the local numbering the pairs share
      if ((s = host_tile_pairs(ne, conn_host, b->order_host, conn_ord))) return s;
    } else {
      for (int64_t p = 0; p < ne; ++p)
        memcpy(&conn_ord[p * b->nnode], conn_host + (int64_t)b->order_host[p] * b->nnode, b->nnode * sizeof(int32_t));
    }
    for (int64_t p = 0; p < ne; ++p) tpos[b->order_host[p]] = (int32_t)p;
    if ((s = b->tpos.upload(tpos.data(), std::max<size_t>(tpos.size(), 1)))) return s;
    if ((s = b->order_dev.upload(b->order_host.data(), std::max<size_t>(b->order_host.size(), 1)))) return s;
    if ((s = b->conn_tile.upload(conn_ord.data(), std::max<size_t>(conn_ord.size(), 1)))) return s;
    std::vector<int32_t> tp, tn;
    std::vector<uint16_t> te, tq;
    if ((s = host_tile_maps(nn, ne, b->nnode, conn_ord.data(), b->tile, tp, tn, te, tq, b->maxu))) return s;
    b->ntile = (int64_t)tp.size() - 1;
    if ((s = b->tile_ptr.upload(tp.data(), tp.size()))) return s;
    if ((s = b->tile_nodes.upload(tn.data(), std::max<size_t>(tn.size(), 1)))) return s;
    if ((s = b->tile_nodes_bc.upload(tn.data(), std::max<size_t>(tn.size(), 1)))) return s;
    b->tile_nodes_host = tn;
    if ((s = b->tile_nend.upload(te.data(), std::max<size_t>(te.size(), 1)))) return s;
    if ((s = b->tile_perm.upload(tq.data(), std::max<size_t>(tq.size(), 1)))) return s;
    {  // forward map of the slot lists: list position of every slot's node
      std::vector<uint16_t> li(tq.size(), 0);
      const int NS = b->nnode * b->tile;
      for (int64_t t = 0; t < b->ntile; ++t) {
        int q = 0;
        for (int k = 0; k < tp[t + 1] - tp[t]; ++k)
          for (; q < te[tp[t] + k]; ++q) li[t * NS + tq[t * NS + q]] = (uint16_t)k;
      }
      if ((s = b->lidx.upload(li.data(), std::max<size_t>(li.size(), 1)))) return s;
    }
    {
      // destinations of the tile sums: a node listed by one tile only is written
      // to y directly by that tile (0x80000000 | node); the others' tile sums go
      // to a compact node-major partials array (node runs in node order, tile
      // order inside a run) that the node pass adds up; that pass covers every
      // node not listed exactly once (multi-tile and unreferenced nodes)
      std::vector<int32_t> occ(nn, 0);
      for (int32_t n : tn) ++occ[n];
      std::vector<int32_t> mlist, mptr(1, 0), start(nn, -1);
      for (int64_t n = 0; n < nn; ++n)
        if (occ[n] != 1) {
          start[n] = mptr.back();
          mlist.push_back((int32_t)n);
          mptr.push_back(mptr.back() + occ[n]);
        }
      std::vector<int32_t> dest(tn.size());
      for (size_t q = 0; q < tn.size(); ++q) {                 // entries in tile order
        const int32_t n = tn[q];
        dest[q] = occ[n] == 1 ? (int32_t)(0x80000000u | (uint32_t)n) : start[n]++;
      }
      b->tile_dest_host = dest;
      b->nmulti = (int64_t)mlist.size();
      if (mlist.empty()) mlist.push_back(0);                   // keep the buffers non-empty
      if (dest.empty()) dest.push_back(0);
      if ((s = b->multi_nodes.upload(mlist.data(), mlist.size()))) return s;
      if ((s = b->multi_nodes_bc.upload(mlist.data(), mlist.size()))) return s;
      b->multi_nodes_host = mlist;
      if ((s = b->multi_ptr.upload(mptr.data(), mptr.size()))) return s;
      if ((s = b->tile_dest.upload(dest.data(), dest.size()))) return s;
      if ((s = b->tile_dest_bc.upload(dest.data(), dest.size()))) return s;
      if ((s = b->partial.alloc(std::max<size_t>(4 * (size_t)mptr.back(), 4)))) return s;   // (x, y, z, 0) per entry
    }
    if ((s = b->dev_err.alloc(1))) return s;
    EX_CUDA(cudaMemset(b->dev_err.p, 0, sizeof(int)));
  }
  if ((s = b->X.upload(X_host, 3 * nn))) return s;
  if ((s = b->conn.upload(conn_host, ne * b->nnode))) return s;
  if ((s = b->plan.upload(b->plan_host.data(), b->plan_host.size()))) return s;
  if ((s = b->colour_elems.upload(elems.data(), elems.size()))) return s;
  if ((s = build_geometry(b.get()))) return s;
  if ((s = init_tangent(b.get()))) return s;
  // element-vector scratch (force assembly, stored-Ke products, diagonals); allocated
  // here so that no later call allocates inside a captured CUDA graph
  if ((s = b->ys.alloc(std::max<int64_t>(ne * b->nnode * 3, 1)))) return s;
  *out = b.release();
  return EXFEM_OK;
} catch (...) {
  return host_exception();
}

int exfem_block_destroy(exfem_block b) {
  delete b;
  return EXFEM_OK;
}

int exfem_block_query(exfem_block b, int64_t* ne, int64_t* nn, int* nnode, int* ngp, int* nstate, int* vmax,
                      int* ncolour, int* affine, int64_t* device_bytes) {
  EX_ARG(b, "block is NULL");
  if (ne) *ne = b->ne;
  if (nn) *nn = b->nn;
  if (nnode) *nnode = b->nnode;
  if (ngp) *ngp = b->ngp;
  if (nstate) *nstate = b->nstate;
  if (vmax) *vmax = b->vmax;
  if (ncolour) *ncolour = b->ncolour;
  if (affine) *affine = b->affine;
  if (device_bytes)
    *device_bytes = (int64_t)(b->X.bytes() + b->conn.bytes() + b->scale.bytes() + b->plan.bytes() +
                              b->colour_elems.bytes() + b->fixed.bytes() + b->node_fixed.bytes() +
                              b->geo64.bytes() + b->geo32.bytes() + b->tan64.bytes() + b->tan32.bytes() +
                              b->ys.bytes());
  return EXFEM_OK;
}

int exfem_block_gather_plan(exfem_block b, int32_t* plan_host) {
  EX_ARG(b && plan_host, "NULL argument");
  memcpy(plan_host, b->plan_host.data(), b->plan_host.size() * sizeof(int32_t));
  return EXFEM_OK;
}

int exfem_block_colours(exfem_block b, int32_t* colour_host) {
  EX_ARG(b && colour_host, "NULL argument");
  memcpy(colour_host, b->colour_host.data(), b->colour_host.size() * sizeof(int32_t));
  return EXFEM_OK;
}

int exfem_block_tile_info(exfem_block b, int64_t* ntile, int64_t* nlist, int* maxu) {
  EX_ARG(b, "block is NULL");
  if (ntile) *ntile = b->ntile;
  if (nlist) {
    int32_t last = 0;
    if (b->ntile) EX_CUDA(cudaMemcpy(&last, b->tile_ptr.p + b->ntile, sizeof(int32_t), cudaMemcpyDeviceToHost));
    *nlist = last;
  }
  if (maxu) *maxu = b->maxu;
  return EXFEM_OK;
}

int exfem_block_tile_maps(exfem_block b, int32_t* ptr_host, int32_t* nodes_host, uint16_t* nend_host,
                          uint16_t* perm_host) {
  EX_ARG(b, "block is NULL");
  int64_t nl = 0;
  int st;
  if ((st = exfem_block_tile_info(b, nullptr, &nl, nullptr))) return st;
  if (ptr_host) EX_CUDA(cudaMemcpy(ptr_host, b->tile_ptr.p, (b->ntile + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (nodes_host && nl) EX_CUDA(cudaMemcpy(nodes_host, b->tile_nodes.p, nl * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (nend_host && nl) EX_CUDA(cudaMemcpy(nend_host, b->tile_nend.p, nl * sizeof(uint16_t), cudaMemcpyDeviceToHost));
  if (perm_host && b->ntile)
    EX_CUDA(cudaMemcpy(perm_host, b->tile_perm.p, (size_t)b->ntile * b->nnode * b->tile * sizeof(uint16_t),
                       cudaMemcpyDeviceToHost));
  return EXFEM_OK;
}

int exfem_block_tile_order(exfem_block b, int* tile, int32_t* order_host) {
  EX_ARG(b, "block is NULL");
  if (tile) *tile = b->tile;
  if (order_host && b->ne) memcpy(order_host, b->order_host.data(), b->ne * sizeof(int32_t));
  return EXFEM_OK;
}

int exfem_block_tile_conn(exfem_block b, int32_t* conn_tile_host) {
  EX_ARG(b && conn_tile_host, "NULL argument");
  if (b->ne)
    EX_CUDA(cudaMemcpy(conn_tile_host, b->conn_tile.p, (size_t)b->ne * b->nnode * sizeof(int32_t),
                       cudaMemcpyDeviceToHost));
  return EXFEM_OK;
}

int exfem_set_tile(int etype, int tile) {
  EX_ARG(etype == EXFEM_C3D8 || etype == EXFEM_C3D10, "unknown element type %d", etype);
  EX_ARG(tile == 128 || tile == 256, "tile size must be 128 or 256, got %d", tile);
  g_tile[etype == EXFEM_C3D8 ? 0 : 1] = tile;
  return EXFEM_OK;
}

int exfem_get_tile(int etype, int* tile) {
  EX_ARG(etype == EXFEM_C3D8 || etype == EXFEM_C3D10, "unknown element type %d", etype);
  EX_ARG(tile, "tile is NULL");
  *tile = g_tile[etype == EXFEM_C3D8 ? 0 : 1];
  return EXFEM_OK;
}

int exfem_block_set_scale(exfem_block b, const double* scale_host) {
  EX_ARG(b, "block is NULL");
  int s;
  if (scale_host) {
    if ((s = b->scale.upload(scale_host, b->ne))) return s;
  } else {
    b->scale.release();
  }
  ++b->bc_gen;
  return build_geometry(b);
}

int exfem_block_set_lame(exfem_block b, const double* lam_host, const double* mu_host) {
  EX_ARG(b, "block is NULL");
  EX_ARG((lam_host == nullptr) == (mu_host == nullptr), "give both Lame arrays or neither");
  EX_ARG(b->mat.kind == EXFEM_LINEAR_ELASTIC || !lam_host, "per-element Lame parameters apply to linear elasticity");
  int s;
  if (lam_host) {
    for (int64_t e = 0; e < b->ne; ++e)
      EX_ARG(mu_host[e] > 0 && lam_host[e] > -2.0 / 3.0 * mu_host[e], "invalid Lame parameters at element %lld",
             (long long)e);
    if ((s = b->lam_e.upload(lam_host, b->ne))) return s;
    if ((s = b->mu_e.upload(mu_host, b->ne))) return s;
  } else {
    b->lam_e.release();
    b->mu_e.release();
  }
  ++b->bc_gen;
  return build_geometry(b);
}

int exfem_block_set_fixed(exfem_block b, const uint8_t* fixed_host) try {
  EX_ARG(b, "block is NULL");
  int s;
  ++b->bc_gen;
  if (!fixed_host) {
    b->fixed.release();
    b->node_fixed.release();
    if (!b->tile_dest_host.empty())
      EX_CUDA(cudaMemcpy(b->tile_dest_bc.p, b->tile_dest_host.data(), b->tile_dest_host.size() * sizeof(int32_t),
                         cudaMemcpyHostToDevice));
    if (!b->multi_nodes_host.empty())
      EX_CUDA(cudaMemcpy(b->multi_nodes_bc.p, b->multi_nodes_host.data(),
                         b->multi_nodes_host.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    if (!b->tile_nodes_host.empty())
      EX_CUDA(cudaMemcpy(b->tile_nodes_bc.p, b->tile_nodes_host.data(), b->tile_nodes_host.size() * sizeof(int32_t),
                         cudaMemcpyHostToDevice));
    return EXFEM_OK;
  }
  std::vector<uint8_t> f(fixed_host, fixed_host + b->ndof()), nf(b->nn, 0);
  for (int64_t n = 0; n < b->nn; ++n)
    for (int c = 0; c < 3; ++c) {
      f[3 * n + c] = f[3 * n + c] ? 1 : 0;
      nf[n] |= (uint8_t)(f[3 * n + c] << c);
    }
  if (!b->multi_nodes_host.empty()) {  // fixed-DOF bits of the node pass's nodes, at bits 28-30
    std::vector<int32_t> packed(b->multi_nodes_host);
    for (auto& q : packed) q = (int32_t)((uint32_t)q | ((uint32_t)nf[q] << 28));
    EX_CUDA(cudaMemcpy(b->multi_nodes_bc.p, packed.data(), packed.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (!b->tile_dest_host.empty()) {   // fixed-DOF bits of nodes written directly, at bits 28-30
    std::vector<int32_t> packed(b->tile_dest_host);
    for (auto& q : packed)
      if (q < 0) q = (int32_t)((uint32_t)q | ((uint32_t)nf[q & 0x0FFFFFFF] << 28));
    EX_CUDA(cudaMemcpy(b->tile_dest_bc.p, packed.data(), packed.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (!b->tile_nodes_host.empty()) {  // fixed-DOF bits packed above the node id
    std::vector<int32_t> packed(b->tile_nodes_host);
    for (auto& q : packed) q = (int32_t)((uint32_t)q | ((uint32_t)nf[q] << 29));
    EX_CUDA(cudaMemcpy(b->tile_nodes_bc.p, packed.data(), packed.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (b->fixed.n == (size_t)b->ndof()) {
    EX_CUDA(cudaMemcpy(b->fixed.p, f.data(), f.size(), cudaMemcpyHostToDevice));
    EX_CUDA(cudaMemcpy(b->node_fixed.p, nf.data(), nf.size(), cudaMemcpyHostToDevice));
    return EXFEM_OK;
  }
  if ((s = b->fixed.upload(f.data(), f.size()))) return s;
  return b->node_fixed.upload(nf.data(), nf.size());
} catch (...) {
  return host_exception();
}

int exfem_internal_force(exfem_block b, const double* u, const double* state_old, double* state_new, double* fe,
                         double* f, int assembly, void* stream) {
  EX_ARG(b && u && f, "NULL argument");
  EX_ARG(b->mat.kind != EXFEM_J2 || state_old, "J2 material needs state_old");
  EX_ARG(assembly == EXFEM_ASSEMBLE_GATHER || assembly == EXFEM_ASSEMBLE_COLOUR, "unknown assembly %d", assembly);
  int s;
  if (!fe) {
    if (b->ys.n < (size_t)(b->ne * b->nnode * 3) && (s = b->ys.alloc(b->ne * b->nnode * 3))) return s;
    fe = b->ys.p;
  }
  if ((s = launch_force(b, FORCE_FULL, u, state_old, state_new, fe, nullptr, nullptr, nullptr, as_stream(stream)))) return s;
  if (b->mat.kind == EXFEM_J2) ++b->tan_gen;
  if (assembly == EXFEM_ASSEMBLE_GATHER) return launch_gather_assemble(b, fe, f, nullptr, nullptr, as_stream(stream));
  return launch_colour_assemble(b, fe, f, as_stream(stream));
}

int exfem_element_stiffness(exfem_block b, const double* u, const double* state_old, int dtype, void* Ke, void* stream) {
  EX_ARG(b && u && Ke, "NULL argument");
  EX_ARG(b->mat.kind != EXFEM_J2 || state_old, "J2 material needs state_old");
  return launch_stiffness(b, u, state_old, dtype, Ke, nullptr, as_stream(stream));
}

int exfem_tangent_update(exfem_block b, const double* u, const double* state_old, void* stream) {
  EX_ARG(b && u, "NULL argument");
  if (b->mat.kind != EXFEM_J2) return EXFEM_OK;
  EX_ARG(state_old, "J2 material needs state_old");
  ++b->tan_gen;
  return launch_force(b, FORCE_TANGENT, u, state_old, nullptr, nullptr, nullptr, nullptr, nullptr, as_stream(stream));
}

int exfem_tangent_matvec(exfem_block b, int dtype, const void* v, void* y, int apply_bc, void* stream) {
  EX_ARG(b && v && y, "NULL argument");
  if (dtype == EXFEM_F64)
    return launch_mf_matvec<double>(b, (const double*)v, (double*)y, nullptr, as_stream(stream), apply_bc != 0);
  if (dtype == EXFEM_F32)
    return launch_mf_matvec<float>(b, (const float*)v, (float*)y, nullptr, as_stream(stream), apply_bc != 0);
  set_error("tangent matvec supports F64 and F32, got %d", dtype);
  return EXFEM_ERR_ARG;
}

int exfem_tangent_diagonal(exfem_block b, double* diag, void* stream) {
  EX_ARG(b && diag, "NULL argument");
  return launch_mf_diagonal(b, diag, as_stream(stream));
}

int exfem_ebe_matvec_bf16_multi(exfem_block b, const void* Ke_bf16, int nrhs, const float* V, float* Y,
                                int apply_bc, void* stream) {
  EX_ARG(b && (b->ne == 0 || Ke_bf16) && V && Y, "NULL argument");
  StreamGuard g;
  int s;
  if ((s = g.init(stream))) return s;
  return launch_ebe_matvec_tc(b, (const __nv_bfloat16*)Ke_bf16, nrhs, V, Y, g.work, apply_bc != 0);
}

int exfem_ebe_matvec_multi(exfem_block b, const void* Ke, int ke_dtype, int nrhs, const void* V, void* Y,
                           int apply_bc, void* stream) {
  EX_ARG(b && (b->ne == 0 || Ke) && V && Y, "NULL argument");
  StreamGuard g;
  int s;
  if ((s = g.init(stream))) return s;
  return launch_ebe_matvec_multi(b, Ke, ke_dtype, nrhs, V, Y, apply_bc != 0, g.work);
}

int exfem_multi_pcg(exfem_block b, const double* Ke, int nrhs, const double* B, double* X, double tol, int maxiter,
                    int* iters, double* relres, void* stream) {
  EX_ARG(b && (b->ne == 0 || Ke) && B && X, "NULL argument");
  EX_ARG(tol > 0 && maxiter >= 0, "tolerance must be positive and maxiter non-negative");
  StreamGuard g;
  int s;
  if ((s = g.init(stream))) return s;
  return multi_pcg(b, Ke, nrhs, B, X, tol, maxiter, iters, relres, g.work);
}

int exfem_ebe_matvec(exfem_block b, const double* Ke, const double* v, double* y, int apply_bc, void* stream) {
  EX_ARG(b && Ke && v && y, "NULL argument");
  return launch_ebe_matvec(b, Ke, v, y, nullptr, as_stream(stream), apply_bc != 0);
}

int exfem_ebe_diagonal(exfem_block b, const double* Ke, double* diag, void* stream) {
  EX_ARG(b && Ke && diag, "NULL argument");
  return launch_ebe_diagonal(b, Ke, diag, as_stream(stream));
}

int exfem_geometric_stiffness(exfem_block b, const double* S, double* Kg, void* stream) {
  EX_ARG(b && (S || b->ne == 0) && (Kg || b->ne == 0), "NULL argument");
  StreamGuard g;
  int st;
  if ((st = g.init(stream))) return st;
  return launch_geo_stiffness(b, S, Kg, g.work);
}

int exfem_stresses(exfem_block b, const double* u, const double* state, double* S, double* mises, double* peeq,
                   void* stream) {
  EX_ARG(b && u, "NULL argument");
  EX_ARG(b->mat.kind != EXFEM_J2 || state, "J2 material needs a state");
  return launch_force(b, FORCE_STRESS, u, state, nullptr, nullptr, S, mises, peeq, as_stream(stream));
}

// ---------------------------------------------------------------- AMG
int exfem_amg_create(exfem_amg* out) {
  EX_ARG(out, "out is NULL");
  *out = new exfem_amg_s();
  return EXFEM_OK;
}

int exfem_amg_destroy(exfem_amg h) {
  delete h;
  return EXFEM_OK;
}

int exfem_amg_add_level(exfem_amg h, int64_t n, int64_t nc, const int64_t* A_ptr, const int32_t* A_idx,
                        const double* A_val, const int64_t* P_ptr, const int32_t* P_idx, const double* P_val,
                        const int64_t* R_ptr, const int32_t* R_idx, const double* R_val, const double* dinv,
                        double rho) try {
  EX_ARG(h && A_ptr && P_ptr && R_ptr && dinv, "NULL argument");
  EX_ARG(n > 0 && nc > 0, "empty level");
  EX_ARG(h->levels.empty() || h->levels.back()->nc == n, "level size %lld does not match the previous coarse size",
         (long long)n);
  EX_ARG(rho > 0 && std::isfinite(rho), "invalid spectral bound %g", rho);
  EX_ARG(!h->replicated, "hierarchy already replicated");
  return amg_add_level(h, n, nc, A_ptr, A_idx, A_val, P_ptr, P_idx, P_val, R_ptr, R_idx, R_val, dinv, rho);
} catch (...) {
  return host_exception();
}

int exfem_amg_set_coarse(exfem_amg h, int64_t nc, const double* Ainv) {
  EX_ARG(h && Ainv, "NULL argument");
  EX_ARG(!h->replicated, "hierarchy already replicated");
  EX_ARG(h->levels.empty() || h->levels.back()->nc == nc, "coarse size mismatch");
  h->nc = nc;
  h->crow_s.release();
  h->crow_m.release();
  h->crow_a.release();
  return h->Ainv.upload(Ainv, (size_t)(nc * nc));
}

int exfem_amg_set_level_rows(exfem_amg h, int level, const double* rho_rows) {
  EX_ARG(h && rho_rows, "NULL argument");
  EX_ARG(!h->replicated, "hierarchy already replicated");
  EX_ARG(level >= 0, "negative level");
  return amg_set_level_rows(h, (size_t)level, rho_rows);
}

int exfem_amg_set_coarse_blocks(exfem_amg h, int64_t nblk, const int64_t* offsets, const double* Ainv_blocks) try {
  EX_ARG(h && offsets && Ainv_blocks && nblk > 0, "NULL argument or no blocks");
  EX_ARG(!h->replicated, "hierarchy already replicated");
  const int64_t nc = offsets[nblk];
  EX_ARG(offsets[0] == 0 && nc > 0, "block offsets must start at 0 and cover at least one row");
  EX_ARG(h->levels.empty() || h->levels.back()->nc == nc, "coarse size mismatch");
  std::vector<int64_t> rs(nc), rm(nc), ra(nc);
  int64_t a = 0;
  for (int64_t b = 0; b < nblk; ++b) {
    const int64_t s0 = offsets[b], m = offsets[b + 1] - s0;
    EX_ARG(m > 0, "empty coarse block %lld", (long long)b);
    for (int64_t r = s0; r < s0 + m; ++r) { rs[r] = s0; rm[r] = m; ra[r] = a; }
    a += m * m;
  }
  int st;
  h->nc = nc;
  if ((st = h->Ainv.upload(Ainv_blocks, (size_t)a))) return st;
  if ((st = h->crow_s.upload(rs.data(), nc))) return st;
  if ((st = h->crow_m.upload(rm.data(), nc))) return st;
  return h->crow_a.upload(ra.data(), nc);
} catch (...) {
  return host_exception();
}

int exfem_amg_replicate(exfem_amg h, int nblk, const int64_t* level_offsets, int ninst, const int32_t* inst_block) {
  EX_ARG(h && level_offsets && inst_block, "NULL argument");
  EX_ARG(nblk >= 1 && ninst >= 1, "need at least one block and one instance");
  EX_ARG(!h->replicated, "hierarchy already replicated");
  return amg_replicate(h, nblk, level_offsets, ninst, inst_block);
}

int exfem_amg_vcycle(exfem_amg h, int dtype, const void* r, void* z, exfem_block level0, const void* dinv0,
                     void* stream) {
  EX_ARG(h && r && z, "NULL argument");
  EX_ARG(!level0 || dinv0, "a level-0 block needs dinv0");
  if (dtype == EXFEM_F64) {
    Level0Op<double> op;
    if (level0) { op.apply = &mf_apply_cb<double>; op.ctx = level0; op.dinv = (const double*)dinv0; }
    return amg_vcycle<double>(h, (const double*)r, (double*)z, level0 ? &op : nullptr, nullptr, as_stream(stream));
  }
  if (dtype == EXFEM_F32) {
    Level0Op<float> op;
    if (level0) { op.apply = &mf_apply_cb<float>; op.ctx = level0; op.dinv = (const float*)dinv0; }
    return amg_vcycle<float>(h, (const float*)r, (float*)z, level0 ? &op : nullptr, nullptr, as_stream(stream));
  }
  set_error("V-cycle supports F64 and F32, got %d", dtype);
  return EXFEM_ERR_ARG;
}

// ---------------------------------------------------------------- solvers
int exfem_solver_create(exfem_block b, int op_kind, int pc_kind, exfem_amg amg, exfem_solver* out) try {
  EX_ARG(b && out, "NULL argument");
  *out = nullptr;
  EX_ARG(op_kind >= EXFEM_OP_EBE_F64 && op_kind <= EXFEM_OP_CSR_F64, "unknown operator kind %d", op_kind);
  EX_ARG(pc_kind >= EXFEM_PC_NONE && pc_kind <= EXFEM_PC_CHEBY, "unknown preconditioner %d", pc_kind);
  EX_ARG(pc_kind != EXFEM_PC_AMG || amg, "AMG preconditioner needs a hierarchy");
  EX_ARG(pc_kind != EXFEM_PC_AMG || amg->levels.empty() || amg->levels[0]->n == b->ndof(),
         "hierarchy level 0 has %lld rows, block has %lld DOFs", (long long)(amg->levels.empty() ? 0 : amg->levels[0]->n),
         (long long)b->ndof());
  auto S = std::make_unique<exfem_solver_s>();
  S->blk = b;
  S->amg = amg;
  S->op = op_kind;
  S->pc = pc_kind;
  S->n = b->ndof();
  int s;
  if ((s = solver_alloc(S.get()))) return s;
  *out = S.release();
  return EXFEM_OK;
} catch (...) {
  return host_exception();
}

int exfem_solver_destroy(exfem_solver s) {
  delete s;
  return EXFEM_OK;
}

int exfem_solver_set_ke(exfem_solver s, const double* Ke) {
  return exfem_solver_set_ke_block(s, 0, Ke);
}

int exfem_solver_add_block(exfem_solver s, exfem_block b) {
  EX_ARG(s && b, "NULL argument");
  EX_ARG(b->nn == s->blk->nn, "an added block must share the solver's node set (%lld vs %lld nodes)",
         (long long)b->nn, (long long)s->blk->nn);
  for (auto& ge : s->gexec)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  s->more.push_back(b);
  s->more_Ke.push_back(nullptr);
  s->diag_ready = false;
  s->csr_dirty = true;
  return EXFEM_OK;
}

int exfem_solver_set_ke_block(exfem_solver s, int block, const double* Ke) {
  EX_ARG(s, "solver is NULL");
  EX_ARG(block >= 0 && block <= (int)s->more.size(), "block %d out of range (the solver has %zu)", block,
         s->more.size() + 1);
  if (block == 0) s->Ke = Ke;
  else s->more_Ke[block - 1] = Ke;
  s->diag_ready = false;
  // EXFEM_OP_CSR_F64: assembled by the next solve, with the prescribed DOFs then in force
  if (s->op == EXFEM_OP_CSR_F64) s->csr_dirty = true;
  return EXFEM_OK;
}

int exfem_solver_refresh_diagonal(exfem_solver s, void* stream) {
  EX_ARG(s, "solver is NULL");
  return solver_refresh_diagonal(s, as_stream(stream));
}

int exfem_solver_cheby_bound(exfem_solver s, double* lmax) {
  EX_ARG(s && lmax, "NULL argument");
  *lmax = s->cheb_lmax;
  return EXFEM_OK;
}

int exfem_solver_set_graph(exfem_solver s, int enable, int chunk) {
  EX_ARG(s, "solver is NULL");
  EX_ARG(chunk >= 1 && chunk <= 1024, "chunk must be in 1..1024");
  for (auto& g : s->gexec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (s->gmixed) { cudaGraphExecDestroy(s->gmixed); s->gmixed = nullptr; }
  s->use_graph = enable ? 1 : 0;
  s->chunk = chunk;
  return EXFEM_OK;
}

int exfem_solver_set_loop(exfem_solver s, int device_loop) {
  EX_ARG(s, "solver is NULL");
  for (auto& g : s->gexec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (s->gmixed) { cudaGraphExecDestroy(s->gmixed); s->gmixed = nullptr; }
  s->device_loop = device_loop ? 1 : 0;
  return EXFEM_OK;
}

int exfem_solver_pcg(exfem_solver s, const double* b, double* x, double tol, int maxiter, int* iters, double* relres,
                     void* stream) {
  EX_ARG(s && b && x, "NULL argument");
  EX_ARG(tol >= 0 && maxiter >= 0, "invalid tolerance or iteration limit");
  StreamGuard g;
  int st;
  if ((st = g.init(stream))) return st;
  const int r = solver_pcg(s, b, x, tol, maxiter, iters, relres, g.work);
  if (r < 0) return r;
  const int w = block_wait_status(s->blk, g.work);
  return w < 0 ? w : r;
}

int exfem_solver_mixed(exfem_solver s, const double* b, double* x, double tol, double inner_tol, int max_pass,
                       int maxiter, int* iters, int* passes, double* relres, void* stream) {
  EX_ARG(s && b && x, "NULL argument");
  EX_ARG(tol >= 0 && inner_tol > 0 && max_pass >= 1 && maxiter >= 0, "invalid refinement parameters");
  StreamGuard g;
  int st;
  if ((st = g.init(stream))) return st;
  // reliable updates run as one graph when the PCG loop runs on the device
  const int r = s->mixed_mode == 1
                    ? (s->use_graph && s->device_loop
                           ? solver_mixed_graph(s, b, x, tol, s->mixed_delta, 100 * max_pass, maxiter, iters, passes,
                                                relres, g.work)
                           : solver_mixed_ru(s, b, x, tol, s->mixed_delta, 100 * max_pass, maxiter, iters, passes,
                                             relres, g.work))
                    : solver_mixed(s, b, x, tol, inner_tol, max_pass, maxiter, iters, passes, relres, g.work);
  if (r < 0) return r;
  const int w = block_wait_status(s->blk, g.work);
  return w < 0 ? w : r;
}

int exfem_newton_increment(exfem_solver s, const double* u, const double* const* states_old, const double* fext,
                           const double* start, double rtol, int max_iter, int line_search, double cg_tol,
                           int cg_maxiter, double* qref, double* u_out, double* const* states_out, int* corrections,
                           int* converged, double* ratios, int* lin_stats, void* stream) {
  EX_ARG(s && u && fext && start && qref && u_out, "NULL argument");
  EX_ARG(rtol > 0 && cg_tol > 0 && cg_maxiter >= 0, "invalid tolerances");
  EX_ARG(s->mixed_mode == 1 && s->use_graph && s->device_loop,
         "the device Newton increment runs the reliable-update mixed solve with graphs and the device loop");
  StreamGuard g;
  int st;
  if ((st = g.init(stream))) return st;
  const int r = newton_increment(s, u, states_old, fext, start, rtol, max_iter, line_search != 0, cg_tol, cg_maxiter,
                                 qref, u_out, states_out, corrections, converged, ratios, lin_stats, g.work);
  if (r < 0) return r;
  const int w = block_wait_status(s->blk, g.work);
  return w < 0 ? w : r;
}

int exfem_solver_set_mixed_mode(exfem_solver s, int mode, double delta) {
  EX_ARG(s, "solver is NULL");
  EX_ARG(mode == 0 || mode == 1, "mixed mode must be 0 (restarted refinement) or 1 (reliable updates)");
  EX_ARG(delta > 0 && delta < 1, "reliable-update reduction must lie in (0, 1), got %g", delta);
  s->mixed_mode = mode;
  s->mixed_delta = delta;
  return EXFEM_OK;
}

int exfem_block_status(exfem_block b, void* stream) {
  EX_ARG(b, "block is NULL");
  StreamGuard g;
  int st;
  if ((st = g.init(stream))) return st;
  return block_wait_status(b, g.work);
}

int exfem_amg_setup_block(exfem_amg h, exfem_block b, const double* Ke, int max_coarse, int keep_level0,
                          void* stream) {
  EX_ARG(h && b, "NULL handle");
  return exfem_amg_setup_blocks(h, 1, &b, &Ke, max_coarse, keep_level0, stream);
}

int exfem_amg_setup_blocks(exfem_amg h, int nblk, const exfem_block* blocks, const double* const* Kes,
                           int max_coarse, int keep_level0, void* stream) try {
  EX_ARG(h && nblk >= 1 && blocks && Kes, "NULL argument");
  std::vector<exfem_block_s*> bl(blocks, blocks + nblk);
  std::vector<const double*> ke(Kes, Kes + nblk);
  for (int i = 0; i < nblk; ++i) EX_ARG(bl[i], "block %d is NULL", i);
  StreamGuard g;
  int st;
  if ((st = g.init(stream))) return st;
  st = amg_setup_blocks(h, bl, ke, max_coarse, keep_level0, g.work);
  if (st) {  // leave the handle empty rather than half built
    h->levels.clear();
    h->nc = 0;
    h->coarse_nnz = 0;
    h->Ainv.release();
  }
  return st;
} catch (...) {
  return host_exception();
}

int exfem_amg_export_level(exfem_amg h, int level, int what, int64_t* rows, int64_t* cols, int64_t* nnz,
                           int64_t* ptr, int32_t* idx, double* val, double* rho) {
  EX_ARG(h && rows && cols && nnz, "NULL argument");
  EX_ARG(level >= 0 && level < (int)h->levels.size(), "level %d out of range", level);
  EX_ARG(!h->replicated, "replicated hierarchies are not exported");
  EX_ARG(what >= 0 && what <= 3, "what must be 0 (A), 1 (P), 2 (R) or 3 (inverse diagonal)");
  const AmgLevel& L = *h->levels[level];
  if (rho) *rho = L.rho;
  if (what == 3) {
    *rows = L.n;
    *cols = 1;
    *nnz = L.n;
    if (val && L.n) EX_CUDA(cudaMemcpy(val, L.dinv64.p, sizeof(double) * L.n, cudaMemcpyDeviceToHost));
    return EXFEM_OK;
  }
  const Csr64& M = what == 0 ? L.A : what == 1 ? L.P : L.R;
  *rows = M.n;
  *cols = M.ncols;
  *nnz = M.nnz;
  if (ptr) {
    if (M.ptr.p) EX_CUDA(cudaMemcpy(ptr, M.ptr.p, sizeof(int64_t) * (M.n + 1), cudaMemcpyDeviceToHost));
    else std::fill(ptr, ptr + M.n + 1, (int64_t)0);
  }
  if (idx && M.nnz) EX_CUDA(cudaMemcpy(idx, M.idx.p, sizeof(int32_t) * M.nnz, cudaMemcpyDeviceToHost));
  if (val && M.nnz) EX_CUDA(cudaMemcpy(val, M.v64.p, sizeof(double) * M.nnz, cudaMemcpyDeviceToHost));
  return EXFEM_OK;
}

int exfem_amg_export_coarse(exfem_amg h, int64_t* nc, double* Ainv) {
  EX_ARG(h && nc, "NULL argument");
  EX_ARG(!h->replicated && !h->crow_s.p, "block-diagonal coarsest solves are not exported");
  *nc = h->nc;
  if (Ainv && h->nc) EX_CUDA(cudaMemcpy(Ainv, h->Ainv.p, sizeof(double) * h->nc * h->nc, cudaMemcpyDeviceToHost));
  return EXFEM_OK;
}

int exfem_amg_info(exfem_amg h, int cap, int* nlevels, int64_t* rows, int64_t* nnz) {
  EX_ARG(h && nlevels, "NULL argument");
  const int nl = (int)h->levels.size() + (h->nc > 0 ? 1 : 0);
  *nlevels = nl;
  for (int l = 0; l < nl && l < cap; ++l) {
    if (l < (int)h->levels.size()) {
      const auto& L = *h->levels[l];
      if (rows) rows[l] = L.n;
      if (nnz) nnz[l] = L.A.nnz ? L.A.nnz : L.op_nnz;
    } else {
      if (rows) rows[l] = h->nc;
      if (nnz) nnz[l] = h->coarse_nnz ? h->coarse_nnz : h->nc * h->nc;
    }
  }
  return EXFEM_OK;
}

int exfem_selftest_bounded_wait(int polls, void* stream) {
  EX_ARG(polls > 0, "polls must be positive");
  DevBuf<int> flag;
  int s;
  if ((s = flag.alloc(1))) return s;
  StreamGuard g;
  if ((s = g.init(stream))) return s;
  EX_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), g.work));
  if ((s = launch_wait_selftest(polls, flag.p, g.work))) return s;
  int h = 0;
  EX_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, g.work));
  EX_CUDA(cudaStreamSynchronize(g.work));
  if (h) {
    set_error("bounded wait gave up after %d polls (expected: nothing arrives in the self-test)", polls);
    return EXFEM_ERR_TIMEOUT;
  }
  return EXFEM_OK;
}

// ---------------------------------------------------------------- host builders
int exfem_host_gather_plan(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int32_t* plan, int* vmax) {
  EX_ARG(conn && vmax, "NULL argument");
  EX_ARG(nn >= 0 && ne >= 0 && nnode >= 0, "invalid sizes (nn %lld, ne %lld, nnode %d)", (long long)nn,
         (long long)ne, nnode);
  return host_guard([&]() -> int {
    std::vector<int32_t> p;
    int v = 0, s;
    if ((s = host_gather_plan(nn, ne, nnode, conn, plan ? &p : nullptr, v))) return s;
    *vmax = v;
    if (plan) memcpy(plan, p.data(), p.size() * sizeof(int32_t));
    return EXFEM_OK;
  });
}

int exfem_host_colouring(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int32_t* colour, int* ncolour) {
  EX_ARG(conn && colour && ncolour, "NULL argument");
  EX_ARG(nn >= 0 && ne >= 0 && nnode >= 0, "invalid sizes (nn %lld, ne %lld, nnode %d)", (long long)nn,
         (long long)ne, nnode);
  for (int64_t k = 0; k < ne * nnode; ++k)
    EX_ARG(conn[k] >= 0 && conn[k] < nn, "connectivity entry %d at slot %lld is outside [0, %lld)", conn[k],
           (long long)k, (long long)nn);
  return host_guard([&]() -> int {
    std::vector<int32_t> c;
    int s;
    if ((s = host_colouring(nn, ne, nnode, conn, c, *ncolour))) return s;
    memcpy(colour, c.data(), c.size() * sizeof(int32_t));
    return EXFEM_OK;
  });
}

int exfem_host_node_adjacency(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int64_t* nnz, int64_t* ptr,
                              int32_t* idx) {
  EX_ARG(nn >= 0 && ne >= 0 && nnode > 0 && (ne == 0 || conn) && nnz && ptr, "invalid arguments");
  return host_guard([&]() -> int {
    Rows r;
    int st;
    if ((st = host_node_adjacency(nn, ne, nnode, conn, r))) return st;
    *nnz = (int64_t)r.idx.size();
    std::copy(r.ptr.begin(), r.ptr.end(), ptr);
    if (idx) std::copy(r.idx.begin(), r.idx.end(), idx);
    return EXFEM_OK;
  });
}

int exfem_host_fit_candidates(int64_t nb, int bs, int K, const int32_t* agg, int64_t nagg, const double* B,
                              double* Q, double* Bc) {
  EX_ARG(nb >= 0 && bs > 0 && K > 0 && nagg >= 0 && agg && B && Q && Bc, "invalid arguments");
  for (int64_t n = 0; n < nb; ++n)
    EX_ARG(agg[n] >= 0 && agg[n] < nagg, "aggregate %d of node %lld out of range", agg[n], (long long)n);
  return host_guard([&]() -> int {
    std::vector<double> q, bc;
    host_fit_candidates(nb, bs, K, agg, nagg, B, q, bc);
    std::copy(q.begin(), q.end(), Q);
    std::copy(bc.begin(), bc.end(), Bc);
    return EXFEM_OK;
  });
}

int exfem_host_coarse_inverse(int64_t n, const double* A, double* Ainv) {
  EX_ARG(n > 0 && n <= (int64_t(1) << 20) && A && Ainv, "invalid arguments");
  return host_guard([&]() -> int {
    std::vector<double> a(A, A + n * n), inv;
    int st;
    if ((st = host_coarse_inverse(n, a, inv))) return st;
    std::copy(inv.begin(), inv.end(), Ainv);
    return EXFEM_OK;
  });
}

int exfem_host_filter_pattern(int64_t nrows, const int64_t* ptr, const int32_t* idx, const uint8_t* flag,
                              int64_t* nnz, int64_t* ptr_out, int32_t* idx_out, int64_t* keep_out) {
  EX_ARG(nrows >= 0 && ptr && nnz, "NULL argument or negative row count");
  EX_ARG(ptr[0] == 0, "ptr[0] must be 0");
  for (int64_t r = 0; r < nrows; ++r) EX_ARG(ptr[r + 1] >= ptr[r], "ptr decreases at row %lld", (long long)r);
  EX_ARG(ptr[nrows] == 0 || (idx && flag), "NULL idx or flag");
  return host_guard([&]() -> int {
    int64_t c = 0;
    for (int64_t q = 0; q < ptr[nrows]; ++q) c += flag[q] ? 1 : 0;
    *nnz = c;
    if (!idx_out) return EXFEM_OK;
    EX_ARG(ptr_out && (keep_out || c == 0), "NULL output");
    Rows pat, S;
    std::vector<int64_t> keep;
    pat.ptr.assign(ptr, ptr + nrows + 1);
    pat.idx.assign(idx, idx + ptr[nrows]);
    host_filter_pattern(pat, flag, S, keep);
    std::copy(S.ptr.begin(), S.ptr.end(), ptr_out);
    std::copy(S.idx.begin(), S.idx.end(), idx_out);
    std::copy(keep.begin(), keep.end(), keep_out);
    return EXFEM_OK;
  });
}

int exfem_host_standard_aggregation(int64_t n, const int64_t* ptr, const int32_t* idx, int32_t* agg, int64_t* nagg) {
  EX_ARG(ptr && idx && agg && nagg, "NULL argument");
  EX_ARG(n >= 0, "negative size %lld", (long long)n);
  return host_guard([&]() -> int { return host_standard_aggregation(n, ptr, idx, agg, *nagg); });
}

int exfem_host_tile_maps(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int tile, int64_t* ntile,
                         int64_t* nlist, int32_t* ptr, int32_t* nodes, uint16_t* nend, uint16_t* perm) {
  EX_ARG(nn >= 0 && ne >= 0 && nnode > 0 && (conn || ne == 0) && ntile && nlist, "NULL argument or invalid sizes");
  EX_ARG(tile == 128 || tile == 256, "tile must be 128 or 256, got %d", tile);
  for (int64_t k = 0; k < ne * nnode; ++k)
    EX_ARG(conn[k] >= 0 && conn[k] < nn, "connectivity entry %d at slot %lld is outside [0, %lld)", conn[k],
           (long long)k, (long long)nn);
  return host_guard([&]() -> int {
    std::vector<int32_t> tp, tn;
    std::vector<uint16_t> te, tq;
    int maxu = 0, s;
    if ((s = host_tile_maps(nn, ne, nnode, conn, tile, tp, tn, te, tq, maxu))) return s;
    *ntile = (int64_t)tp.size() - 1;
    *nlist = (int64_t)tn.size();
    if (ptr) memcpy(ptr, tp.data(), tp.size() * sizeof(int32_t));
    if (nodes) memcpy(nodes, tn.data(), tn.size() * sizeof(int32_t));
    if (nend) memcpy(nend, te.data(), te.size() * sizeof(uint16_t));
    if (perm) memcpy(perm, tq.data(), tq.size() * sizeof(uint16_t));
    return EXFEM_OK;
  });
}

int exfem_host_face_once(int64_t nface, const int64_t* keys, uint8_t* once) {
  EX_ARG(nface >= 0 && ((keys && once) || nface == 0), "NULL argument");
  return host_guard([&]() -> int { return host_face_once(nface, keys, once); });
}

int exfem_host_tile_pairs(int64_t ne, const int32_t* conn, int32_t* order, int32_t* conn_tile) {
  EX_ARG(ne >= 0 && (conn || ne == 0) && (order || ne == 0) && (conn_tile || ne == 0), "NULL argument");
  return host_guard([&]() -> int {
    std::vector<char> seen(ne, 0);
    for (int64_t k = 0; k < ne; ++k) {
      EX_ARG(order[k] >= 0 && order[k] < ne && !seen[order[k]], "order is not a permutation of [0, %lld) at %lld",
             (long long)ne, (long long)k);
      seen[order[k]] = 1;
    }
    std::vector<int32_t> o(order, order + ne), ct;
    int s;
    if ((s = host_tile_pairs(ne, conn, o, ct))) return s;
    if (ne) {
      memcpy(order, o.data(), ne * sizeof(int32_t));
      memcpy(conn_tile, ct.data(), ct.size() * sizeof(int32_t));
    }
    return EXFEM_OK;
  });
}

int exfem_host_tile_order(int64_t nn, int64_t ne, int nnode, int ncorner, const double* X, const int32_t* conn,
                          int32_t* order) {
  EX_ARG(nn >= 0 && ne >= 0 && nnode > 0 && ncorner > 0 && ncorner <= nnode, "invalid sizes");
  EX_ARG((X || nn == 0) && (conn || ne == 0) && (order || ne == 0), "NULL argument");
  for (int64_t k = 0; k < ne * nnode; ++k)
    EX_ARG(conn[k] >= 0 && conn[k] < nn, "connectivity entry %d at slot %lld is outside [0, %lld)", conn[k],
           (long long)k, (long long)nn);
  return host_guard([&]() -> int {
    std::vector<int32_t> o;
    int s;
    if ((s = host_tile_order(nn, ne, nnode, ncorner, X, conn, o))) return s;
    if (ne) memcpy(order, o.data(), ne * sizeof(int32_t));
    return EXFEM_OK;
  });
}

}  // extern "C"
