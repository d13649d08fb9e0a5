// Host-side index builders of the exfem_b200 library (no device work).
//
//  * gather plan (gfem/model.py:241-261): for every node, the flat element
//    slots elem*nnode + local that touch it, in increasing slot order (the
//    reference's stable argsort by node), padded with the sentinel ne*nnode to
//    the maximum valence.  Built here with a counting sort; bit-identical.
//  * greedy element colouring (no counterpart in the reference): elements in
//    index order take the smallest colour unused by every element that shares a
//    node with them.
//  * standard aggregation for smoothed aggregation (Vanek, Mandel & Brezina,
//    "Algebraic multigrid by smoothed aggregation", 1996; PyAMG's default
//    'standard' aggregation, which the reference calls through
//    pyamg.smoothed_aggregation_solver at gfem/linalg.py:113-116):
//      pass 1: every node whose strong neighbours are all unaggregated seeds an
//              aggregate with them; nodes with no neighbour stay unaggregated;
//      pass 2: remaining nodes join the first neighbouring pass-1 aggregate;
//      pass 3: still-unaggregated nodes seed new aggregates with their
//              unaggregated neighbours.
//  * tile maps of the matrix-free product: per tile of consecutive positions of
//    the tile order, its sorted distinct nodes and the slots grouped by node
//    (tiles in parallel);
//  * boundary faces (no counterpart in the reference's code, which finds them
//    with a row-wise np.unique, gfem/surfaces.py:182-221): every element face
//    is keyed by its sorted corner nodes; the keys go into an open-addressing hash
//    table (linear probing, power-of-two size at least twice the face count)
//    that counts equal keys; a face is on the boundary when its key occurs once.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace exfem {

int host_gather_plan(int64_t nn, int64_t ne, int nnode, const int32_t* conn, std::vector<int32_t>* plan_out,
                     int& vmax) {
  const int64_t nslot = ne * nnode;
  for (int64_t k = 0; k < nslot; ++k) {
    const int32_t n = conn[k];
    if (n < 0 || n >= nn) {
      set_error("connectivity entry %d at slot %lld is outside [0, %lld)", n, (long long)k, (long long)nn);
      return EXFEM_ERR_ARG;
    }
  }
  if (nslot >= (int64_t)INT32_MAX) {
    set_error("gather plan needs int64 slots (ne*nnode >= 2^31)");
    return EXFEM_ERR_UNSUPPORTED;
  }
  // threads own contiguous node ranges and each scans every slot in increasing
  // order, so a row lists its slots in increasing order exactly as one counting
  // sort does, and each thread's counters and plan rows stay within its range
  const int nth = (int)std::max<int64_t>(
      1, std::min<int64_t>(std::min<int>((int)std::thread::hardware_concurrency(), 16), nslot / (1 << 20)));
  std::vector<int32_t> cnt(nn, 0);
  auto range = [&](int t, int64_t& lo, int64_t& hi) {
    lo = nn * t / nth;
    hi = nn * (t + 1) / nth;
  };
  auto run = [&](auto&& f) {
    if (nth == 1) { f(0); return; }
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; ++t) pool.emplace_back(f, t);
    for (auto& th : pool) th.join();
  };
  run([&](int t) {
    int64_t lo, hi;
    range(t, lo, hi);
    for (int64_t k = 0; k < nslot; ++k) {
      const int32_t n = conn[k];
      if (n >= lo && n < hi) ++cnt[n];
    }
  });
  int32_t m = 1;
  for (int64_t n = 0; n < nn; ++n) m = cnt[n] > m ? cnt[n] : m;
  vmax = m;
  if (!plan_out) return EXFEM_OK;  // the width alone
  std::vector<int32_t>& plan = *plan_out;
  plan.resize((size_t)nn * vmax);
  run([&](int t) {
    int64_t lo, hi;
    range(t, lo, hi);
    std::fill(plan.begin() + lo * vmax, plan.begin() + hi * vmax, (int32_t)nslot);
    std::fill(cnt.begin() + lo, cnt.begin() + hi, 0);
    for (int64_t k = 0; k < nslot; ++k) {
      const int32_t n = conn[k];
      if (n >= lo && n < hi) plan[(size_t)n * vmax + cnt[n]++] = (int32_t)k;
    }
  });
  return EXFEM_OK;
}

int host_colouring(int64_t nn, int64_t ne, int nnode, const int32_t* conn, std::vector<int32_t>& colour,
                   int& ncolour) {
  constexpr int W = 4;  // 256 colours
  std::vector<uint64_t> used((size_t)nn * W, 0);
  colour.assign(ne, 0);
  ncolour = 0;
  for (int64_t e = 0; e < ne; ++e) {
    uint64_t m[W] = {0, 0, 0, 0};
    for (int a = 0; a < nnode; ++a) {
      const int64_t n = conn[e * nnode + a];
      for (int w = 0; w < W; ++w) m[w] |= used[n * W + w];
    }
    int c = 0;
    while (c < 64 * W && ((m[c >> 6] >> (c & 63)) & 1ull)) ++c;
    if (c >= 64 * W) {
      set_error("element colouring needs more than %d colours", 64 * W);
      return EXFEM_ERR_UNSUPPORTED;
    }
    colour[e] = c;
    if (c + 1 > ncolour) ncolour = c + 1;
    for (int a = 0; a < nnode; ++a) {
      const int64_t n = conn[e * nnode + a];
      used[n * W + (c >> 6)] |= (1ull << (c & 63));
    }
  }
  return EXFEM_OK;
}

// Tile order of the matrix-free operator (no counterpart in the reference):
// elements are grouped by connected component (components in the order of their
// first element) and, inside a component, sorted along a Morton (Z-order) curve
// of their corner-node coordinate sums, ties by element index.  Consecutive
// positions are then spatially compact, so a tile of consecutive positions
// touches few distinct nodes, and the tiles of one mesh never mix with another
// mesh of the same union block.  The key:
//   s_e   = x_{c0} + x_{c1} + ... (corner nodes in local order, summed in order)
//   q_e,d = min(floor((s_e,d - lo_d) / (hi_d - lo_d) * 2^21), 2^21 - 1)
//           (0 when hi_d == lo_d), lo/hi the extent of s over all elements
//   key   = bits of q_x, q_y, q_z interleaved (x lowest).
int host_tile_order(int64_t nn, int64_t ne, int nnode, int ncorner, const double* X, const int32_t* conn,
                    std::vector<int32_t>& order) {
  order.resize(ne);
  if (ne == 0) return EXFEM_OK;
  // components: union-find over the nodes of each element
  std::vector<int32_t> parent(nn);
  for (int64_t n = 0; n < nn; ++n) parent[n] = (int32_t)n;
  auto find = [&](int32_t a) {
    while (parent[a] != a) {
      parent[a] = parent[parent[a]];
      a = parent[a];
    }
    return a;
  };
  for (int64_t e = 0; e < ne; ++e) {
    int32_t r0 = find(conn[e * nnode]);
    for (int a = 1; a < nnode; ++a) {
      const int32_t r = find(conn[e * nnode + a]);
      if (r < r0) {
        parent[r0] = r;
        r0 = r;
      } else if (r > r0) {
        parent[r] = r0;
      }
    }
  }
  std::vector<int64_t> first(nn, -1), comp(ne);
  for (int64_t e = 0; e < ne; ++e) {
    const int32_t r = find(conn[e * nnode]);
    if (first[r] < 0) first[r] = e;
    comp[e] = first[r];
  }
  std::vector<double> s((size_t)ne * 3);
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int64_t e = 0; e < ne; ++e)
    for (int d = 0; d < 3; ++d) {
      double v = X[3 * (int64_t)conn[e * nnode] + d];
      for (int a = 1; a < ncorner; ++a) v += X[3 * (int64_t)conn[e * nnode + a] + d];
      s[3 * e + d] = v;
      if (e == 0 || v < lo[d]) lo[d] = v;
      if (e == 0 || v > hi[d]) hi[d] = v;
    }
  // sort records (component, Morton key, element): the order is strict, so chunks
  // sorted by separate threads and merged give the one sorted sequence
  struct Rec {
    int64_t comp;
    uint64_t key;
    int32_t e;
    bool operator<(const Rec& o) const {
      if (comp != o.comp) return comp < o.comp;
      if (key != o.key) return key < o.key;
      return e < o.e;
    }
  };
  std::vector<Rec> rec(ne);
  const int nth = (int)std::max<int64_t>(
      1, std::min<int64_t>(std::min<int>((int)std::thread::hardware_concurrency(), 16), ne / (1 << 16)));
  std::vector<int64_t> cut(nth + 1);
  for (int t = 0; t <= nth; ++t) cut[t] = ne * t / nth;
  auto chunk = [&](int t) {
    for (int64_t e = cut[t]; e < cut[t + 1]; ++e) {
      uint64_t k = 0;
      for (int d = 0; d < 3; ++d) {
        uint64_t q = 0;
        if (hi[d] > lo[d]) {
          const double f = std::floor((s[3 * e + d] - lo[d]) / (hi[d] - lo[d]) * 2097152.0);
          q = f >= 2097151.0 ? 2097151u : (f > 0.0 ? (uint64_t)f : 0u);
        }
        for (int b = 0; b < 21; ++b) k |= ((q >> b) & 1ull) << (3 * b + d);
      }
      rec[e] = Rec{comp[e], k, (int32_t)e};
    }
    std::sort(rec.begin() + cut[t], rec.begin() + cut[t + 1]);
  };
  if (nth == 1) {
    chunk(0);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; ++t) pool.emplace_back(chunk, t);
    for (auto& th : pool) th.join();
    // pairwise merges of neighbouring runs, the merges of one round in parallel
    for (int w = 1; w < nth; w *= 2) {
      std::vector<std::thread> mp;
      for (int t = 0; t + w < nth; t += 2 * w) {
        const int64_t a = cut[t], m = cut[t + w], b = cut[std::min(t + 2 * w, nth)];
        mp.emplace_back([&rec, a, m, b]() { std::inplace_merge(rec.begin() + a, rec.begin() + m, rec.begin() + b); });
      }
      for (auto& th : mp) th.join();
    }
  }
  for (int64_t p = 0; p < ne; ++p) order[p] = rec[p].e;
  return EXFEM_OK;
}

// Face pairs of the C3D10 tile order (no counterpart in the reference).  The
// FP32 product evaluates the elements at positions 2j and 2j+1 in one thread; when
// the two share a face, their three shared corners and three shared edge nodes are
// loaded and accumulated once if they sit at fixed local positions: corners
// (p, q, r) of the face at local 0, 1, 2 of the first element and at 1, 0, 2 of the
// second (so local 0<->1, 1<->0, 2<->2 and edge nodes 4<->4, 5<->6, 6<->5), the
// other corner last.  Both stay positively oriented: the first element is an even
// permutation of its corners with the non-shared corner last, the second is
// (q, p, r, t), which is even for a valid mesh (t lies on the other side of the
// face); if it is not, the pair keeps its elements' own numbering.
//   pairing: walking the tile order, every element not yet placed takes the first
//   unplaced element sharing three corners with it among the next 16 positions;
//   the pairs and the remaining single elements keep the order of their first
//   element, and consecutive singles are put side by side.
// Returns the new order and the connectivity of every position in the local
// numbering used by the tiles (mid-edge nodes follow their corners).
static const int TET_EDGES[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};

static int tet_edge_of(int a, int b) {
  for (int k = 0; k < 6; ++k)
    if ((TET_EDGES[k][0] == a && TET_EDGES[k][1] == b) || (TET_EDGES[k][0] == b && TET_EDGES[k][1] == a)) return k;
  return -1;
}

static bool even_perm(const int* p) {
  int inv = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = i + 1; j < 4; ++j) inv += p[i] > p[j];
  return (inv & 1) == 0;
}

// new local corner i = old local corner pi[i]; writes the element's 10 nodes
static void tet10_permuted(const int32_t* c, const int* pi, int32_t* out) {
  for (int i = 0; i < 4; ++i) out[i] = c[pi[i]];
  for (int k = 0; k < 6; ++k) out[4 + k] = c[4 + tet_edge_of(pi[TET_EDGES[k][0]], pi[TET_EDGES[k][1]])];
}

int host_tile_pairs(int64_t ne, const int32_t* conn, std::vector<int32_t>& order, std::vector<int32_t>& conn_tile) {
  constexpr int W = 16;
  std::vector<char> used(ne, 0);
  std::vector<std::pair<int32_t, int32_t>> units;
  units.reserve(ne);
  auto shared = [&](int32_t e, int32_t f) {
    int n = 0;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) n += conn[e * 10 + i] == conn[f * 10 + j];
    return n;
  };
  for (int64_t k = 0; k < ne; ++k) {
    const int32_t e = order[k];
    if (used[e]) continue;
    used[e] = 1;
    int32_t mate = -1;
    for (int64_t m = k + 1; m < ne && m <= k + W; ++m) {
      const int32_t f = order[m];
      if (!used[f] && shared(e, f) == 3) {
        mate = f;
        break;
      }
    }
    if (mate >= 0) used[mate] = 1;
    units.push_back({e, mate});
  }
  order.clear();
  conn_tile.assign((size_t)ne * 10, 0);
  auto emit = [&](int32_t e, const int* pi) {
    const int64_t p = (int64_t)order.size();
    order.push_back(e);
    if (pi) tet10_permuted(conn + (int64_t)e * 10, pi, conn_tile.data() + p * 10);
    else memcpy(conn_tile.data() + p * 10, conn + (int64_t)e * 10, 10 * sizeof(int32_t));
  };
  int32_t pending = -1;
  for (const auto& u : units) {
    if (u.second < 0) {
      if (pending < 0) {
        pending = u.first;
      } else {
        emit(pending, nullptr);
        emit(u.first, nullptr);
        pending = -1;
      }
      continue;
    }
    const int32_t* ce = conn + (int64_t)u.first * 10;
    const int32_t* cf = conn + (int64_t)u.second * 10;
    int se = -1, tf = -1;                       // local index of the corner off the shared face
    for (int i = 0; i < 4; ++i) {
      bool in_f = false, in_e = false;
      for (int j = 0; j < 4; ++j) {
        in_f |= ce[i] == cf[j];
        in_e |= cf[i] == ce[j];
      }
      if (!in_f) se = i;
      if (!in_e) tf = i;
    }
    int pe[4] = {0, 1, 2, 3}, pf[4];
    bool ok = false;
    do {                                          // first even permutation (lexicographic) with se last
      if (pe[3] == se && even_perm(pe)) { ok = true; break; }
    } while (std::next_permutation(pe, pe + 4));
    if (ok) {
      const int32_t want[4] = {ce[pe[1]], ce[pe[0]], ce[pe[2]], cf[tf]};   // (q, p, r, t)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          if (cf[j] == want[i]) pf[i] = j;
      ok = even_perm(pf);
    }
    if (ok) {
      emit(u.first, pe);
      emit(u.second, pf);
    } else {
      emit(u.first, nullptr);
      emit(u.second, nullptr);
    }
  }
  if (pending >= 0) emit(pending, nullptr);
  return EXFEM_OK;
}

// Element-tile maps of the matrix-free operator.  Tiles are `tile` consecutive
// positions of the tile order (conn is given in that order), and slot
// s = a*tile + p is local node a of the element at tile position p.  Per tile:
// the sorted distinct nodes it touches; for each of them, in node order, its
// slots in increasing slot order, concatenated into `perm` (tile-major, padded
// to nnode*tile entries per tile); and `nend`, the end of each node's run in
// perm (aligned with the node list).
int host_tile_maps(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int tile, std::vector<int32_t>& ptr, std::vector<int32_t>& nodes, std::vector<uint16_t>& nend,
                   std::vector<uint16_t>& perm, int& maxu) {
  const int64_t ntile = (ne + tile - 1) / tile;
  const int nslot = nnode * tile;
  ptr.assign(ntile + 1, 0);
  nend.clear();
  perm.assign((size_t)ntile * nslot, 0);
  // per tile: the sorted distinct nodes (independent per tile, so the tiles are
  // processed in parallel and concatenated in tile order)
  std::vector<std::vector<int32_t>> lists(ntile);
  std::vector<std::vector<uint16_t>> ends(ntile);
  const int nth = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 16));
  std::vector<std::thread> pool;
  std::atomic<int64_t> next_tile(0);
  auto work = [&]() {
    std::vector<int32_t> pos(nn, 0), cntv, start;
    for (;;) {
      const int64_t t = next_tile.fetch_add(1);
      if (t >= ntile) break;
      const int64_t e0 = t * tile, e1 = std::min<int64_t>(ne, e0 + tile);
      std::vector<int32_t> list(conn + e0 * nnode, conn + e1 * nnode);
      std::sort(list.begin(), list.end());
      list.erase(std::unique(list.begin(), list.end()), list.end());
      const int nu = (int)list.size();
      for (int i = 0; i < nu; ++i) pos[list[i]] = i;
      cntv.assign(nu, 0);
      for (int a = 0; a < nnode; ++a)
        for (int64_t e = e0; e < e1; ++e) ++cntv[pos[conn[e * nnode + a]]];
      start.assign(nu + 1, 0);
      for (int i = 0; i < nu; ++i) start[i + 1] = start[i] + cntv[i];
      uint16_t* pm = perm.data() + (size_t)t * nslot;
      for (int i = 0; i < nu; ++i) cntv[i] = start[i];
      for (int a = 0; a < nnode; ++a)                      // increasing slot order
        for (int64_t e = e0; e < e1; ++e) pm[cntv[pos[conn[e * nnode + a]]]++] = (uint16_t)(a * tile + (e - e0));
      std::vector<uint16_t> en(nu);
      for (int i = 0; i < nu; ++i) en[i] = (uint16_t)start[i + 1];
      lists[t] = std::move(list);
      ends[t] = std::move(en);
    }
  };
  for (int i = 0; i < nth; ++i) pool.emplace_back(work);
  for (auto& th : pool) th.join();
  nodes.clear();
  maxu = 0;
  for (int64_t t = 0; t < ntile; ++t) {
    nodes.insert(nodes.end(), lists[t].begin(), lists[t].end());
    nend.insert(nend.end(), ends[t].begin(), ends[t].end());
    ptr[t + 1] = (int32_t)nodes.size();
    maxu = std::max<int>(maxu, (int)lists[t].size());
  }
  return EXFEM_OK;
}

int host_standard_aggregation(int64_t n, const int64_t* ptr, const int32_t* idx, int32_t* agg, int64_t& nagg) {
  constexpr int32_t UNSET = -2, ISOLATED = -1;
  std::vector<uint8_t> seeded(n, 0);  // 1 = member of a pass-1 aggregate
  for (int64_t i = 0; i < n; ++i) agg[i] = UNSET;
  int32_t next = 0;
  for (int64_t i = 0; i < n; ++i) {  // pass 1
    if (agg[i] != UNSET) continue;
    bool has_nb = false, free_nbs = true;
    for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
      const int64_t j = idx[k];
      if (j == i) continue;
      has_nb = true;
      if (agg[j] != UNSET) { free_nbs = false; break; }
    }
    if (!has_nb) {
      agg[i] = ISOLATED;
    } else if (free_nbs) {
      agg[i] = next;
      seeded[i] = 1;
      for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
        agg[idx[k]] = next;
        seeded[idx[k]] = 1;
      }
      ++next;
    }
  }
  for (int64_t i = 0; i < n; ++i) {  // pass 2
    if (agg[i] != UNSET) continue;
    for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
      const int64_t j = idx[k];
      if (j != i && seeded[j]) { agg[i] = agg[j]; break; }
    }
  }
  for (int64_t i = 0; i < n; ++i) {  // pass 3
    if (agg[i] != UNSET) continue;
    agg[i] = next;
    for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
      if (agg[idx[k]] == UNSET) agg[idx[k]] = next;
    ++next;
  }
  nagg = next;
  return EXFEM_OK;
}

static inline uint64_t face_key_hash(const int64_t* k) {
  uint64_t h = 0x9e3779b97f4a7c15ull;
  for (int i = 0; i < 4; ++i) {  // splitmix64 steps over the four key words
    uint64_t z = h + (uint64_t)k[i] + 0x9e3779b97f4a7c15ull * (uint64_t)(i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    h = z ^ (z >> 31);
  }
  return h;
}

int host_face_once(int64_t nface, const int64_t* keys, uint8_t* once) {
  if (nface == 0) return EXFEM_OK;
  size_t cap = 1;
  while (cap < 2 * (size_t)nface) cap <<= 1;
  std::vector<int64_t> slot(cap, -1);   // first face holding each distinct key
  std::vector<int32_t> count(nface, 0);
  std::vector<int64_t> first(nface);
  for (int64_t f = 0; f < nface; ++f) {
    const int64_t* k = keys + 4 * f;
    size_t h = (size_t)face_key_hash(k) & (cap - 1);
    for (;;) {
      const int64_t g = slot[h];
      if (g < 0) { slot[h] = f; first[f] = f; break; }
      const int64_t* kg = keys + 4 * g;
      if (kg[0] == k[0] && kg[1] == k[1] && kg[2] == k[2] && kg[3] == k[3]) { first[f] = g; break; }
      h = (h + 1) & (cap - 1);
    }
    ++count[first[f]];
  }
  for (int64_t f = 0; f < nface; ++f) once[f] = count[first[f]] == 1 ? 1 : 0;
  return EXFEM_OK;
}

}  // namespace exfem
