// Host-side triangle-mesh connectivity: EToE/EToF and the vmapM/vmapP node
// maps, bit-exact with ddg's src/ddg/dg2d/mesh.py:520-627.  The reference
// builds vmapP with a Python double loop over K x 3 faces; here it is one
// pass in C++ (the dominant host cost of admitting a new mesh).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

#include "../../include/ddg_sipg.h"
#include "status.h"

extern "C" int ddg_mesh_connect(int64_t K, const int64_t* EToV, int64_t* EToE, int64_t* EToF) {
  if (K <= 0 || !EToV || !EToE || !EToF) return ddg::fail(DDG_ERR_INVALID, "ddg_mesh_connect: bad arguments");
  int64_t nn = 0;
  for (int64_t i = 0; i < 3 * K; ++i) {
    if (EToV[i] < 0) return ddg::fail(DDG_ERR_INVALID, "ddg_mesh_connect: negative vertex id");
    nn = std::max(nn, EToV[i] + 1);
  }
  // Face g = f*K + k (all faces 0, then 1, then 2: mesh.py:548-551).
  const int64_t nf = 3 * K;
  std::vector<int64_t> key(nf);
  for (int f = 0; f < 3; ++f)
    for (int64_t k = 0; k < K; ++k) {
      int64_t a = EToV[k * 3 + f], b = EToV[k * 3 + (f + 1) % 3];
      if (a > b) std::swap(a, b);
      key[f * K + k] = a * nn + b;
    }
  std::vector<int64_t> order(nf);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return key[x] < key[y]; });
  for (int64_t k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) { EToE[k * 3 + f] = k; EToF[k * 3 + f] = f; }
  // Adjacent equal keys pair up, in sorted order (mesh.py:561-570).
  for (int64_t i = 0; i + 1 < nf; ++i) {
    if (key[order[i]] != key[order[i + 1]]) continue;
    const int64_t g1 = order[i], g2 = order[i + 1];
    const int64_t k1 = g1 % K, f1 = g1 / K, k2 = g2 % K, f2 = g2 / K;
    EToE[k1 * 3 + f1] = k2; EToF[k1 * 3 + f1] = f2;
    EToE[k2 * 3 + f2] = k1; EToF[k2 * 3 + f2] = f1;
  }
  return DDG_OK;
}

extern "C" int ddg_mesh_maps(int64_t K, int32_t N, const int64_t* Fmask, const double* x,
                             const double* y, const int64_t* EToE, const int64_t* EToF,
                             const int64_t* EToV, const double* VX, const double* VY,
                             double node_tol, int64_t* vmapM, int64_t* vmapP) {
  if (K <= 0 || N < 0 || !Fmask || !x || !y || !EToE || !EToF || !EToV || !VX || !VY || !vmapM || !vmapP)
    return ddg::fail(DDG_ERR_INVALID, "ddg_mesh_maps: bad arguments");
  const int Nfp = N + 1, Np = (N + 1) * (N + 2) / 2;
  // x, y are (Np, K) row-major; the flat F-order index of (n, k) is k*Np + n.
  auto X = [&](int64_t id) { return x[(id % Np) * K + id / Np]; };
  auto Y = [&](int64_t id) { return y[(id % Np) * K + id / Np]; };
  // vmapM[(k*3 + f)*Nfp + p] = k*Np + Fmask[p, f]   (mesh.py:594-596)
  for (int64_t k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f)
      for (int p = 0; p < Nfp; ++p) {
        const int64_t fm = Fmask[p * 3 + f];
        if (fm < 0 || fm >= Np) return ddg::fail(DDG_ERR_INVALID, "ddg_mesh_maps: Fmask out of range");
        vmapM[(k * 3 + f) * Nfp + p] = k * Np + fm;
      }
  std::vector<double> xm(Nfp), ym(Nfp), xp(Nfp), yp(Nfp);
  for (int64_t k1 = 0; k1 < K; ++k1)
    for (int f1 = 0; f1 < 3; ++f1) {
      const int64_t k2 = EToE[k1 * 3 + f1], f2 = EToF[k1 * 3 + f1];
      if (k2 < 0 || k2 >= K || f2 < 0 || f2 > 2) return ddg::fail(DDG_ERR_INVALID, "ddg_mesh_maps: bad EToE/EToF");
      const int64_t v1 = EToV[k1 * 3 + f1], v2 = EToV[k1 * 3 + (f1 + 1) % 3];
      const double ref_d = std::sqrt((VX[v1] - VX[v2]) * (VX[v1] - VX[v2]) + (VY[v1] - VY[v2]) * (VY[v1] - VY[v2]));
      const int64_t* idM = vmapM + (k1 * 3 + f1) * Nfp;
      const int64_t* idP = vmapM + (k2 * 3 + f2) * Nfp;
      for (int p = 0; p < Nfp; ++p) { xm[p] = X(idM[p]); ym[p] = Y(idM[p]); xp[p] = X(idP[p]); yp[p] = Y(idP[p]); }
      for (int p = 0; p < Nfp; ++p) {
        int64_t hit = idM[p];                                  // boundary fallback
        for (int q = 0; q < Nfp; ++q) {
          const double dx = xm[p] - xp[q], dy = ym[p] - yp[q];
          if (std::sqrt(dx * dx + dy * dy) < node_tol * ref_d) { hit = idP[q]; break; }
        }
        vmapP[(k1 * 3 + f1) * Nfp + p] = hit;
      }
    }
  return DDG_OK;
}
