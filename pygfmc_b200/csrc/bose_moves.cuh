// The Bose-Hubbard move layout on the device, shared by the step kernels:
// decode of an off-diagonal slot and its element before the guide.
#pragma once
#include <cstdint>

#include "engine.cuh"

namespace gfmc {

// ---- Bose-Hubbard transition layout (bose_hubbard.py module docstring;
//      _common.two_site_move:34-72) -------------------------------------------
struct BoseMove {
  int a, b, da, db, blk, idx;  // blk: 0 hop fwd, 1 hop bwd, 2 pair up, 3 pair dn, 4 b+, 5 b
};

template <typename T>
__device__ __forceinline__ BoseMove bose_decode(const DevModel<T> &m, int o) {
  BoseMove mv;
  int E = m.E;
  if (m.n_hop) {
    if (o < 2 * E) {
      int e = o < E ? o : o - E;
      uint32_t pe = m.edge[e];
      mv.a = pe & 0xFFFF; mv.b = pe >> 16; mv.idx = e;
      if (o < E) { mv.da = -1; mv.db = +1; mv.blk = 0; }
      else { mv.da = +1; mv.db = -1; mv.blk = 1; }
      return mv;
    }
    o -= 2 * E;
  }
  if (m.n_eta) {
    if (o < 2 * E) {
      int e = o < E ? o : o - E;
      uint32_t pe = m.edge[e];
      mv.a = pe & 0xFFFF; mv.b = pe >> 16; mv.idx = e;
      if (o < E) { mv.da = +1; mv.db = +1; mv.blk = 2; }
      else { mv.da = -1; mv.db = -1; mv.blk = 3; }
      return mv;
    }
    o -= 2 * E;
  }
  int k = o < m.N ? o : o - m.N;
  mv.a = mv.b = k; mv.idx = k; mv.db = 0;
  if (o < m.N) { mv.da = +1; mv.blk = 4; } else { mv.da = -1; mv.blk = 5; }
  return mv;
}

// Unguided off-diagonal element of a decoded move (BoseHubbard.get_rates:
// 285-393): zero where the cutoff n_max forbids it.
// The square roots of the occupation products (integers up to
// (n_max + 1)^2) come from m.sqrt_tab, filled on the host with the same
// correctly rounded square root.
template <typename T>
__device__ __forceinline__ T bose_element(const DevModel<T> &m, const uint8_t *occ,
                                          const BoseMove &mv) {
  // (occupations clamped to n_max: the table bounds hold even for unchecked input)
  const int nmax = m.n_max;
  const int na = occ[mv.a] < nmax ? occ[mv.a] : nmax, nb = occ[mv.b] < nmax ? occ[mv.b] : nmax;
  switch (mv.blk) {
    case 0: return -m.t[mv.idx] * m.sqrt_tab[na * (nb + 1)] * (nb < nmax ? T(1) : T(0));
    case 1: return -m.t[mv.idx] * m.sqrt_tab[(na + 1) * nb] * (na < nmax ? T(1) : T(0));
    case 2:
      return -m.eta[mv.idx] * m.sqrt_tab[(na + 1) * (nb + 1)] *
             ((na < nmax && nb < nmax) ? T(1) : T(0));
    case 3: return -m.eta[mv.idx] * m.sqrt_tab[na * nb];
    case 4: return m.hpm[mv.idx] * m.sqrt_tab[na + 1] * (na < nmax ? T(1) : T(0));
    default: return m.hpm[mv.idx] * m.sqrt_tab[na];
  }
}

}  // namespace gfmc
