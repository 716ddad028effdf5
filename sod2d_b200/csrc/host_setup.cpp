// Host-side set-up for the SOD2D hot path: GLL tables, node-ordering maps,
// a synthetic periodic cube mesh, Jacobians, lumped mass and element sizes.
// Declarations and the reference routines each function replaces are in
// include/sod2d_host.h.  All arrays use the reference's Fortran layout.
#include "sod2d_host.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

// Legendre polynomial P_N and its first two derivatives by the three-term
// recurrence (Bonnet's formula).
void legendre(int n, double x, double &p, double &dp, double &d2p) {
  double p0 = 1.0, dp0 = 0.0, d2p0 = 0.0;
  if (n == 0) { p = p0; dp = dp0; d2p = d2p0; return; }
  double p1 = x, dp1 = 1.0, d2p1 = 0.0;
  for (int k = 2; k <= n; ++k) {
    double a = (2.0 * k - 1.0) / k, b = (k - 1.0) / k;
    double p2 = a * x * p1 - b * p0;
    double dp2 = a * (p1 + x * dp1) - b * dp0;
    double d2p2 = a * (2.0 * dp1 + x * d2p1) - b * d2p0;
    p0 = p1; dp0 = dp1; d2p0 = d2p1;
    p1 = p2; dp1 = dp2; d2p1 = d2p2;
  }
  p = p1; dp = dp1; d2p = d2p1;
}

// 1-D SOD2D ordering [-1, +1, interior ascending] -> natural (ascending) index.
inline int nat_of(int porder, int ii /*0-based SOD2D index*/) {
  if (ii == 0) return 0;
  if (ii == 1) return porder;
  return ii - 1;
}

// Lagrange basis (and derivative) of the GLL grid, polynomial ii in SOD2D
// order, evaluated at s.  Product formula as in eval_lagrangePoly /
// eval_lagrangePolyDeriv (mod_maths.f90:243-323).
double lagrange(int porder, const double *x, int ii, double s) {
  int c = nat_of(porder, ii);
  double l = 1.0;
  for (int j = 0; j <= porder; ++j)
    if (j != c) l *= (s - x[j]) / (x[c] - x[j]);
  return l;
}
double lagrange_deriv(int porder, const double *x, int ii, double s) {
  int c = nat_of(porder, ii);
  double dl = 0.0;
  for (int j = 0; j <= porder; ++j) {
    if (j == c) continue;
    double aux = 1.0;
    for (int m = 0; m <= porder; ++m)
      if (m != j && m != c) aux *= (s - x[m]) / (x[c] - x[m]);
    dl += (1.0 / (x[c] - x[j])) * aux;
  }
  return dl;
}

inline uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Uniform in [-1, 1) from a counter-based hash of (seed, a, b).
inline double hash_uniform(uint64_t seed, uint64_t a, uint64_t b) {
  uint64_t h = splitmix64(seed ^ splitmix64(a * 0x100000001B3ull + b));
  return ((h >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
}

}  // namespace

extern "C" {

int sod_host_gll(int porder, double *xi, double *w) {
  if (porder < 1 || porder > 16 || !xi || !w) return -1;
  const int n = porder;
  xi[0] = -1.0;
  xi[n] = 1.0;
  // Interior nodes: roots of P_N', by Newton's method on P_N' started from the
  // Chebyshev-Gauss-Lobatto points; symmetric by construction.
  for (int i = 1; i <= (n - 1) / 2 + ((n - 1) % 2); ++i) {
    double x = -std::cos(M_PI * i / n);
    for (int it = 0; it < 100; ++it) {
      double p, dp, d2p;
      legendre(n, x, p, dp, d2p);
      double dx = dp / d2p;
      x -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    xi[i] = x;
    xi[n - i] = -x;
  }
  if (n % 2 == 0) xi[n / 2] = 0.0;
  for (int i = 0; i <= n; ++i) {
    double p, dp, d2p;
    legendre(n, xi[i], p, dp, d2p);
    w[i] = 2.0 / (n * (n + 1.0) * p * p);
  }
  return 0;
}

int sod_host_atoijk(int porder, int kind, uint64_t seed, int *atoIJK) {
  if (porder < 2 || porder > 16 || !atoIJK) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1;
  // Vertices in gmsh order as SOD2D 1-D indices (0 -> xi=-1, 1 -> xi=+1).
  static const int vtx[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  std::vector<int> number(nnode, 0);  // tensor position c -> node number
  auto cpos = [&](int i, int j, int k) { return (k * np1 + i) * np1 + j; };
  for (int v = 0; v < 8; ++v) number[cpos(vtx[v][0], vtx[v][1], vtx[v][2])] = v + 1;
  std::vector<int> rest;
  for (int c = 0; c < nnode; ++c)
    if (number[c] == 0) rest.push_back(c);
  std::vector<int> ids(rest.size());
  for (size_t t = 0; t < ids.size(); ++t) ids[t] = 9 + (int)t;
  if (kind == 1) {
    uint64_t s = seed;
    for (size_t t = ids.size(); t > 1; --t) {
      s = splitmix64(s);
      size_t r = s % t;
      std::swap(ids[t - 1], ids[r]);
    }
  } else if (kind != 0) {
    return -2;
  }
  for (size_t t = 0; t < rest.size(); ++t) number[rest[t]] = ids[t];
  for (int c = 0; c < nnode; ++c) atoIJK[c] = number[c];
  return 0;
}

int sod_host_atoijk_inverse(int porder, const int *atoIJK, int *invAtoIJK,
                            int *gmshAtoI, int *gmshAtoJ, int *gmshAtoK) {
  if (porder < 1 || !atoIJK) return -1;
  const int np1 = porder + 1;
  int c = 0;
  for (int k = 0; k < np1; ++k)
    for (int i = 0; i < np1; ++i)
      for (int j = 0; j < np1; ++j) {
        int a = atoIJK[c++];  // 1-based node number
        if (invAtoIJK) invAtoIJK[i + np1 * (j + np1 * k)] = a;
        if (gmshAtoI) gmshAtoI[a - 1] = i + 1;
        if (gmshAtoJ) gmshAtoJ[a - 1] = j + 1;
        if (gmshAtoK) gmshAtoK[a - 1] = k + 1;
      }
  return 0;
}

int sod_host_shape_tables(int porder, const int *atoIJK, float *xgp, float *wgp,
                          float *Ngp, float *dNgp, float *dlxigp_ip) {
  if (porder < 1 || porder > 16 || !atoIJK) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1, ngaus = nnode;
  double x[17], w[17];
  sod_host_gll(porder, x, w);
  // Gauss points: xgp(atoIJK(c),:) = (xi(i), xi(j), xi(k)) over SOD2D order.
  std::vector<float> xg(ngaus * 3);
  std::vector<double> wg(ngaus);
  int c = 0;
  for (int k = 0; k < np1; ++k)
    for (int i = 0; i < np1; ++i)
      for (int j = 0; j < np1; ++j) {
        int a = atoIJK[c++] - 1;
        xg[a + ngaus * 0] = (float)x[nat_of(porder, i)];
        xg[a + ngaus * 1] = (float)x[nat_of(porder, j)];
        xg[a + ngaus * 2] = (float)x[nat_of(porder, k)];
        wg[a] = w[nat_of(porder, i)] * w[nat_of(porder, j)] * w[nat_of(porder, k)];
      }
  if (xgp) std::memcpy(xgp, xg.data(), sizeof(float) * ngaus * 3);
  if (wgp)
    for (int g = 0; g < ngaus; ++g) wgp[g] = (float)wg[g];
  // Shape functions are evaluated at the FP32-rounded Gauss-point coordinates
  // (the reference reads them back from its FP32 xgp array).
  for (int g = 0; g < ngaus; ++g) {
    double s[3];
    for (int d = 0; d < 3; ++d) s[d] = (double)xg[g + ngaus * d];
    double l[3][17], dl[3][17];
    for (int d = 0; d < 3; ++d)
      for (int ii = 0; ii < np1; ++ii) {
        l[d][ii] = lagrange(porder, x, ii, s[d]);
        dl[d][ii] = lagrange_deriv(porder, x, ii, s[d]);
      }
    if (dlxigp_ip)
      for (int ii = 0; ii < np1; ++ii)
        for (int d = 0; d < 3; ++d)
          dlxigp_ip[g + ngaus * (d + 3 * ii)] = (float)dl[d][ii];
    c = 0;
    for (int k = 0; k < np1; ++k)
      for (int i = 0; i < np1; ++i)
        for (int j = 0; j < np1; ++j) {
          int a = atoIJK[c++] - 1;
          if (Ngp) Ngp[g + ngaus * a] = (float)(l[0][i] * l[1][j] * l[2][k]);
          if (dNgp) {
            dNgp[0 + 3 * (a + nnode * g)] = (float)(dl[0][i] * l[1][j] * l[2][k]);
            dNgp[1 + 3 * (a + nnode * g)] = (float)(l[0][i] * dl[1][j] * l[2][k]);
            dNgp[2 + 3 * (a + nnode * g)] = (float)(l[0][i] * l[1][j] * dl[2][k]);
          }
        }
  }
  return 0;
}

int sod_host_cube_sizes(int porder, int nx, int ny, int nz, int *nelem,
                        int *npoin, int *npoin_w) {
  if (porder < 2 || nx < 1 || ny < 1 || nz < 1) return -1;
  long long ne = (long long)nx * ny * nz;
  long long np = (long long)(porder * nx + 1) * (porder * ny + 1) * (porder * nz + 1);
  long long nw = (long long)(porder * nx) * (porder * ny) * (porder * nz);
  if (np > 2000000000LL) return -2;
  if (nelem) *nelem = (int)ne;
  if (npoin) *npoin = (int)np;
  if (npoin_w) *npoin_w = (int)nw;
  return 0;
}

int sod_host_cube_mesh(int porder, int nx, int ny, int nz, double L,
                       double jitter, uint64_t seed, int elem_shuffle,
                       const int *atoIJK, float *coord, int *connecOrig,
                       int *connecWork, int *lpoin_w) {
  int nelem, npoin, npoin_w;
  if (sod_host_cube_sizes(porder, nx, ny, nz, &nelem, &npoin, &npoin_w)) return -1;
  if (!atoIJK || !coord || !connecOrig || !connecWork || !lpoin_w) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1;
  const int gx = porder * nx + 1, gy = porder * ny + 1, gz = porder * nz + 1;
  double x[17], w[17];
  sod_host_gll(porder, x, w);
  const double hx = L / nx, hy = L / ny, hz = L / nz;
  // Per tensor position c: natural 1-D indices and element-local node number.
  std::vector<int> cin(nnode), cjn(nnode), ckn(nnode), cnode(nnode);
  {
    int c = 0;
    for (int k = 0; k < np1; ++k)
      for (int i = 0; i < np1; ++i)
        for (int j = 0; j < np1; ++j, ++c) {
          cin[c] = nat_of(porder, i);
          cjn[c] = nat_of(porder, j);
          ckn[c] = nat_of(porder, k);
          cnode[c] = atoIJK[c] - 1;
        }
  }
  // Grid-point coordinates (FP64), element boundaries at e*h.
  auto gridpos = [&](int g, int ne_, double h) {
    int e = g / porder, r = g % porder;
    if (e == ne_) { e = ne_ - 1; r = porder; }
    return e * h + 0.5 * (x[r] + 1.0) * h;
  };
  std::vector<double> X(gx), Y(gy), Z(gz);
  for (int i = 0; i < gx; ++i) X[i] = gridpos(i, nx, hx);
  for (int i = 0; i < gy; ++i) Y[i] = gridpos(i, ny, hy);
  for (int i = 0; i < gz; ++i) Z[i] = gridpos(i, nz, hz);
  const long long nn = npoin;
  for (int k = 0; k < gz; ++k)
    for (int j = 0; j < gy; ++j)
      for (int i = 0; i < gx; ++i) {
        long long p = i + (long long)gx * (j + (long long)gy * k);
        coord[p + nn * 0] = (float)X[i];
        coord[p + nn * 1] = (float)Y[j];
        coord[p + nn * 2] = (float)Z[k];
      }
  // Element order (optionally shuffled).
  std::vector<int> eorder(nelem);
  for (int e = 0; e < nelem; ++e) eorder[e] = e;
  if (elem_shuffle) {
    uint64_t s = seed ^ 0xA5A5A5A5ull;
    for (int t = nelem; t > 1; --t) {
      s = splitmix64(s);
      std::swap(eorder[t - 1], eorder[s % t]);
    }
  }
  // Local GLL spacing (reference coordinates) for the jitter amplitude.
  double sp[17];
  for (int r = 1; r < porder; ++r) sp[r] = std::min(x[r + 1] - x[r], x[r] - x[r - 1]);
  const long long ne = nelem;
  for (int ie = 0; ie < nelem; ++ie) {
    int eg = eorder[ie];
    int ex = eg % nx, ey = (eg / nx) % ny, ez = eg / (nx * ny);
    for (int c = 0; c < nnode; ++c) {
      int ix = porder * ex + cin[c], iy = porder * ey + cjn[c], iz = porder * ez + ckn[c];
      long long p = ix + (long long)gx * (iy + (long long)gy * iz);
      int wx = ix == gx - 1 ? 0 : ix, wy = iy == gy - 1 ? 0 : iy, wz = iz == gz - 1 ? 0 : iz;
      long long pw = wx + (long long)gx * (wy + (long long)gy * wz);
      connecOrig[ie + ne * cnode[c]] = (int)(p + 1);
      connecWork[ie + ne * cnode[c]] = (int)(pw + 1);
      bool interior = cin[c] > 0 && cin[c] < porder && cjn[c] > 0 && cjn[c] < porder &&
                      ckn[c] > 0 && ckn[c] < porder;
      if (jitter > 0.0 && interior) {
        double dx = jitter * sp[cin[c]] * 0.5 * hx * hash_uniform(seed, (uint64_t)p, 0);
        double dy = jitter * sp[cjn[c]] * 0.5 * hy * hash_uniform(seed, (uint64_t)p, 1);
        double dz = jitter * sp[ckn[c]] * 0.5 * hz * hash_uniform(seed, (uint64_t)p, 2);
        coord[p + nn * 0] = (float)(X[ix] + dx);
        coord[p + nn * 1] = (float)(Y[iy] + dy);
        coord[p + nn * 2] = (float)(Z[iz] + dz);
      }
    }
  }
  long long t = 0;
  for (int k = 0; k < gz - 1; ++k)
    for (int j = 0; j < gy - 1; ++j)
      for (int i = 0; i < gx - 1; ++i)
        lpoin_w[t++] = (int)(i + (long long)gx * (j + (long long)gy * k) + 1);
  return t == npoin_w ? 0 : -3;
}

int sod_host_elem_jacobian(int porder, int nelem, int npoin,
                           const int *connec, const float *coord,
                           const float *dNgp, const float *wgp, float *gpvol,
                           float *He) {
  if (porder < 1 || !connec || !coord || !dNgp || !wgp || !gpvol || !He) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1, ngaus = nnode;
  const long long ne = nelem, nn = npoin;
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < ne; ++e) {
    for (int g = 0; g < ngaus; ++g) {
      double Je[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double dot = 0.0;
          for (int a = 0; a < nnode; ++a) {
            long long p = connec[e + ne * a] - 1;
            float prod = dNgp[i + 3 * (a + (long long)nnode * g)] * coord[p + nn * j];
            dot += (double)prod;
          }
          Je[i][j] = dot;
        }
      double det = Je[0][0] * Je[1][1] * Je[2][2] + Je[0][1] * Je[1][2] * Je[2][0] +
                   Je[0][2] * Je[1][0] * Je[2][1] - Je[2][0] * Je[1][1] * Je[0][2] -
                   Je[2][1] * Je[1][2] * Je[0][0] - Je[2][2] * Je[1][0] * Je[0][1];
      float detf = (float)det;
      double a[9];
      a[0] = Je[1][1] * Je[2][2] - Je[2][1] * Je[1][2];
      a[1] = -(Je[1][0] * Je[2][2] - Je[2][0] * Je[1][2]);
      a[2] = Je[1][0] * Je[2][1] - Je[2][0] * Je[1][1];
      a[3] = -(Je[0][1] * Je[2][2] - Je[2][1] * Je[0][2]);
      a[4] = Je[0][0] * Je[2][2] - Je[2][0] * Je[0][2];
      a[5] = -(Je[0][0] * Je[2][1] - Je[2][0] * Je[0][1]);
      a[6] = Je[0][1] * Je[1][2] - Je[1][1] * Je[0][2];
      a[7] = -(Je[0][0] * Je[1][2] - Je[1][0] * Je[0][2]);
      a[8] = Je[0][0] * Je[1][1] - Je[1][0] * Je[0][1];
      // adjugate = transpose of the cofactor matrix
      double b[9] = {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]};
      double inv = (double)(1.0f / detf);
      float *he = He + 9 * ((long long)g + (long long)ngaus * e);
      // He(i,j) = b(3(i-1)+j), column-major He(3,3,...)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) he[i + 3 * j] = (float)(inv * b[3 * i + j]);
      gpvol[g + (long long)ngaus * e] = wgp[g] * detf;
    }
  }
  return 0;
}

int sod_host_lumped_mass(int porder, int nelem, int npoin, int npoin_w,
                         const int *connec, const int *lpoin_w,
                         const float *gpvol, float *Ml, float *invMl,
                         double *vol_total) {
  if (porder < 1 || !connec || !gpvol || !Ml) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1, ngaus = nnode;
  const long long ne = nelem;
  for (long long p = 0; p < npoin; ++p) Ml[p] = 0.0f;
  double vol = 0.0;
  for (long long e = 0; e < ne; ++e)
    for (int a = 0; a < nnode; ++a) {
      Ml[connec[e + ne * a] - 1] += gpvol[a + ngaus * e];
      vol += (double)gpvol[a + ngaus * e];
    }
  if (invMl) {
    for (long long p = 0; p < npoin; ++p) invMl[p] = 0.0f;
    for (long long t = 0; t < npoin_w; ++t) {
      int p = lpoin_w[t] - 1;
      invMl[p] = 1.0f / Ml[p];
    }
  }
  if (vol_total) *vol_total = vol;
  return 0;
}

int sod_host_char_length(int porder, int nelem, int npoin,
                         const int *connec, const float *coord,
                         float *helem, float *helem_l) {
  if (porder < 1 || !connec || !coord) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1;
  const long long ne = nelem, nn = npoin;
  static const int edges[12][2] = {{1, 0}, {2, 1}, {3, 2}, {0, 3}, {5, 4}, {6, 5},
                                   {7, 6}, {4, 7}, {4, 0}, {5, 1}, {6, 2}, {7, 3}};
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < ne; ++e) {
    if (helem) {
      double xp[8][3];
      for (int v = 0; v < 8; ++v)
        for (int d = 0; d < 3; ++d) xp[v][d] = (double)coord[(connec[e + ne * v] - 1) + nn * d];
      double dmin = 1000000000000.0;
      for (int ed = 0; ed < 12; ++ed) {
        double s = 0.0;
        for (int d = 0; d < 3; ++d) {
          double dd = xp[edges[ed][0]][d] - xp[edges[ed][1]][d];
          s += dd * dd;
        }
        dmin = std::min(dmin, std::sqrt(s));
      }
      helem[e] = (float)dmin;
    }
    if (helem_l) {
      for (int a = 0; a < nnode; ++a) {
        long long pa = connec[e + ne * a] - 1;
        float aux = 1000000000000.0f;
        for (int b = 0; b < nnode; ++b) {
          if (a == b) continue;
          long long pb = connec[e + ne * b] - 1;
          float d0 = coord[pa] - coord[pb];
          float d1 = coord[pa + nn] - coord[pb + nn];
          float d2 = coord[pa + 2 * nn] - coord[pb + 2 * nn];
          float s = d0 * d0 + d1 * d1 + d2 * d2;
          aux = std::min(std::sqrt(s), aux);
        }
        helem_l[e + ne * a] = aux;
      }
    }
  }
  return 0;
}

int sod_host_elem_per_node(int porder, int nelem, int npoin,
                           const int *connec, int *lelpn) {
  if (porder < 1 || !connec || !lelpn) return -1;
  const int np1 = porder + 1, nnode = np1 * np1 * np1;
  const long long ne = nelem;
  for (long long p = 0; p < npoin; ++p) lelpn[p] = 0;
  for (long long e = 0; e < ne; ++e)
    for (int a = 0; a < nnode; ++a) lelpn[connec[e + ne * a] - 1] += 1;
  return 0;
}

int sod_host_tgv_comp_init(int npoin, const float *coord, float Ma, float V0,
                           float L, float T0, float Re, float gamma_gas,
                           float Prt, float *rho, float *u, float *q,
                           float *pr, float *E, float *Tem, float *e_int,
                           float *csound, float *machno, float *eta,
                           float *consts) {
  if (!coord || !rho || !u || !q || !pr || !E || !Tem || !e_int || !csound ||
      !machno || !eta)
    return -1;
  const float g = gamma_gas;
  const float Rgas = V0 * V0 / (g * T0 * Ma * Ma);
  const float Cp = g * Rgas / (g - 1.0f);
  const float rho0 = (1.0f / (g * Ma * Ma)) / (Rgas * T0);
  const float mul = (rho0 * V0 * L) / Re;
  const float P0 = 1.0f / (Ma * Ma * g);
  const float mur = 0.000001458f * std::pow(T0, 1.50f) / (T0 + 110.40f);
  const float mu_factor = mul / mur;
  if (consts) {
    consts[0] = Rgas; consts[1] = Cp; consts[2] = rho0; consts[3] = P0;
    consts[4] = mu_factor; consts[5] = g; consts[6] = Prt; consts[7] = Ma;
  }
  const long long nn = npoin;
#pragma omp parallel for schedule(static)
  for (long long p = 0; p < nn; ++p) {
    float x = coord[p], y = coord[p + nn], z = coord[p + 2 * nn];
    float u0 = V0 * std::sin(x / L) * std::cos(y / L) * std::cos(z / L);
    float u1 = -(V0 * std::cos(x / L) * std::sin(y / L) * std::cos(z / L));
    float u2 = 0.0f;
    float prv = P0 + ((1.0f * V0 * V0) / 16.0f) * (std::cos(2.0f * x / L) + std::cos(2.0f * y / L)) *
                         (std::cos(2.0f * z / L) + 2.0f);
    float r = prv / Rgas / T0;
    u[p] = u0; u[p + nn] = u1; u[p + 2 * nn] = u2;
    pr[p] = prv;
    rho[p] = r;
    float ei = prv / (r * (g - 1.0f));
    e_int[p] = ei;
    Tem[p] = prv / (r * Rgas);
    float uu = u0 * u0 + u1 * u1 + u2 * u2;
    E[p] = r * (0.5f * uu + ei);
    q[p] = r * u0; q[p + nn] = r * u1; q[p + 2 * nn] = r * u2;
    float c = std::sqrt(g * prv / r);
    csound[p] = c;
    machno[p] = uu / c;
    eta[p] = (r / (g - 1.0f)) * std::log(prv / std::pow(r, g));
  }
  return 0;
}

}  // extern "C"
