// The host side of BEST around the solver seam, in C++: what BEST's Fortran driver does before and
// after the hot path, for callers that have no Fortran compiler (and for the benchmarks).  It calls
// the GPU only through the nine bhm_* functions, exactly as best/besolve.f90 does, and keeps the
// Fortran's arithmetic order (sequential sums over triangles, left-to-right expressions), so its
// results match BEST's to rounding.
//
//   best_setup      best/best.f:261-337   centroid shift, areas, area correction, COMPON
//   COMPON          best/compon.f90:19-116
//   deflation       best/best.f:384-404, DEFGAM best/compon.f90:185-197 (XMU, GDEF)
//   rhs6, strain5   best/difco.f:28-44, best/visco.f:216-243
//   difco           best/difco.f:53-401   friction tensors, CR, D_t, D_r, D_tr, CD
//   matin3          best/matin3.f:1-118
//   visco           best/visco.f:24-213   viscosity centre and CHI'
//   jacobi          best/jacobi.f:1-96
//   output          best/output.f:1-176   the .be file
//   run             best/best.f:184-510 + best/besolve.f90:149-240 (HMPREP) as one program
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/best_driver.h"
#include "../../include/best_gpu.h"
#include "../../include/best_hmatrix.h"
#include "bgpu_internal.h"

namespace {

using Mat3 = double[3][3];

// best/best.f:261-315
void setup_arrays(int n, const double* tri, int iarea, double truearea, double* v1, double* v2, double* v3,
                  double* area, double* afac, double* totarea, double* cen) {
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (int t = 0; t < n; ++t) s = s + (tri[9 * (size_t)t + c] + tri[9 * (size_t)t + 3 + c] + tri[9 * (size_t)t + 6 + c]) / 3;
    cen[c] = s / n;
  }
  for (int t = 0; t < n; ++t)
    for (int c = 0; c < 3; ++c) {
      v1[(size_t)c * n + t] = tri[9 * (size_t)t + c] - cen[c];
      v2[(size_t)c * n + t] = tri[9 * (size_t)t + 3 + c] - cen[c];
      v3[(size_t)c * n + t] = tri[9 * (size_t)t + 6 + c] - cen[c];
    }
  double tot = 0.0;
  for (int t = 0; t < n; ++t) {
    const double v21x = v2[t] - v1[t], v21y = v2[n + t] - v1[n + t], v21z = v2[2 * (size_t)n + t] - v1[2 * (size_t)n + t];
    const double v31x = v3[t] - v1[t], v31y = v3[n + t] - v1[n + t], v31z = v3[2 * (size_t)n + t] - v1[2 * (size_t)n + t];
    const double a = v31y * v21z - v31z * v21y, b = v31z * v21x - v31x * v21z, c = v31x * v21y - v31y * v21x;
    area[t] = std::sqrt(a * a + b * b + c * c) * 0.5;
    tot = tot + area[t];
  }
  *totarea = tot;
  if (iarea) {
    *afac = truearea / tot;
    for (int t = 0; t < n; ++t) area[t] = *afac * area[t];
  } else {
    *afac = 1.0;
  }
}

// best/compon.f90:19-116: surfaces of triangles sharing a vertex (exact coordinates); nopen =
// edges not shared by exactly two triangles.
void compon(int n, const double* v1, const double* v2, const double* v3, int* icomp, int* ncomp, int* nopen) {
  const int nv = 3 * n;
  std::vector<std::array<double, 3>> key(nv);
  for (int t = 0; t < n; ++t)
    for (int c = 0; c < 3; ++c) {
      key[3 * t][c] = v1[(size_t)c * n + t];
      key[3 * t + 1][c] = v2[(size_t)c * n + t];
      key[3 * t + 2][c] = v3[(size_t)c * n + t];
    }
  std::vector<int> idx(nv);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key[a] < key[b]; });
  std::vector<int> vid(nv);
  int nid = 0;
  for (int j = 0; j < nv; ++j) {
    if (j == 0 || key[idx[j]] != key[idx[j - 1]]) ++nid;
    vid[idx[j]] = nid;
  }
  std::vector<int> root(n);
  std::iota(root.begin(), root.end(), 0);
  auto find = [&](int i) {
    int p = i;
    while (root[p] != p) p = root[p];
    while (root[i] != p) {
      const int q = root[i];
      root[i] = p;
      i = q;
    }
    return p;
  };
  for (int j = 1; j < nv; ++j)
    if (vid[idx[j]] == vid[idx[j - 1]]) {
      const int a = find(idx[j] / 3), b = find(idx[j - 1] / 3);
      if (a != b) root[std::max(a, b)] = std::min(a, b);
    }
  std::vector<int> lab(n, 0);
  int nc = 0;
  for (int t = 0; t < n; ++t) {
    const int r = find(t);
    if (lab[r] == 0) lab[r] = ++nc;
    icomp[t] = lab[r];
  }
  std::vector<std::pair<int, int>> edges(nv);
  for (int t = 0; t < n; ++t)
    for (int c = 0; c < 3; ++c) {
      const int a = vid[3 * t + c], b = vid[3 * t + (c + 1) % 3];
      edges[3 * t + c] = {std::min(a, b), std::max(a, b)};
    }
  std::sort(edges.begin(), edges.end());
  int open = 0;
  for (int j = 0; j < nv;) {
    int k = j;
    while (k < nv && edges[k] == edges[j]) ++k;
    if (k - j != 2) ++open;
    j = k;
  }
  *ncomp = nc;
  *nopen = open;
}

inline double re(double x) { return x; }
inline double re(const std::complex<double>& x) { return x.real(); }

// best/matin3.f: inverse of a 3x3 by Crout LU with implicit scaling.  a[i][j] = A(i+1, j+1).
// T is double, or std::complex<double> for complex-step derivatives (pivoting on the real parts).
template <class T>
int matin3_t(const T A[3][3], T Y[3][3]) {
  T a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = A[i][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Y[i][j] = (i == j) ? T(1.0) : T(0.0);
  const int n = 3;
  double vv[3];
  int ierr = 0;
  for (int i = 0; i < n; ++i) {
    double aamax = 0.0;
    for (int j = 0; j < n; ++j)
      if (std::fabs(re(a[i][j])) > aamax) aamax = std::fabs(re(a[i][j]));
    if (aamax == 0.0) {
      ierr = 1;
      aamax = 1.0;
    }
    vv[i] = 1.0 / aamax;
  }
  if (ierr) return 1;
  int indx[3] = {0, 0, 0}, imax = 0;
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) {
      T s = a[i][j];
      if (i > 0) {
        for (int k = 0; k < i; ++k) s = s - a[i][k] * a[k][j];
        a[i][j] = s;
      }
    }
    double aamax = 0.0;
    for (int i = j; i < n; ++i) {
      T s = a[i][j];
      if (j > 0) {
        for (int k = 0; k < j; ++k) s = s - a[i][k] * a[k][j];
        a[i][j] = s;
      }
      const double dum = vv[i] * std::fabs(re(s));
      if (dum >= aamax) {
        imax = i;
        aamax = dum;
      }
    }
    if (j != imax) {
      for (int k = 0; k < n; ++k) std::swap(a[imax][k], a[j][k]);
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (j != n - 1) {
      if (re(a[j][j]) == 0.0) a[j][j] = 1e-20;
      const T dum = 1.0 / a[j][j];
      for (int i = j + 1; i < n; ++i) a[i][j] = a[i][j] * dum;
    }
  }
  if (re(a[n - 1][n - 1]) == 0.0) a[n - 1][n - 1] = 1e-20;
  for (int col = 0; col < n; ++col) {
    T b[3] = {Y[0][col], Y[1][col], Y[2][col]};
    int ii = -1;
    for (int i = 0; i < n; ++i) {
      const int ll = indx[i];
      T s = b[ll];
      b[ll] = b[i];
      if (ii != -1) {
        for (int j = ii; j < i; ++j) s = s - a[i][j] * b[j];
      } else if (re(s) != 0.0) {
        ii = i;
      }
      b[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
      T s = b[i];
      for (int j = i + 1; j < n; ++j) s = s - a[i][j] * b[j];
      b[i] = s / a[i][i];
    }
    for (int r = 0; r < n; ++r) Y[r][col] = b[r];
  }
  return 0;
}

int matin3(const Mat3 A, Mat3 Y) { return matin3_t<double>(A, Y); }

void antisym(const double u[3], Mat3 uu) {
  uu[2][0] = -u[1];
  uu[2][1] = u[0];
  uu[0][1] = -u[2];
  uu[1][0] = -uu[0][1];
  uu[1][2] = -uu[2][1];
  uu[0][2] = -uu[2][0];
  uu[0][0] = uu[1][1] = uu[2][2] = 0.0;
}

// best/jacobi.f: eigenvalues of a symmetric 3x3 (upper triangle used), cyclic Jacobi.
void jacobi3(const Mat3 A, double d[3]) {
  double a[3][3], v[3][3], b[3], z[3];
  std::memcpy(a, A, sizeof a);
  const int n = 3;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) v[i][j] = (i == j) ? 1.0 : 0.0;
    b[i] = d[i] = a[i][i];
    z[i] = 0.0;
  }
  for (int it = 1; it <= 50; ++it) {
    double sm = 0.0;
    for (int ip = 0; ip < n - 1; ++ip)
      for (int iq = ip + 1; iq < n; ++iq) sm = sm + std::fabs(a[ip][iq]);
    if (sm == 0.0) return;
    const double tresh = it < 4 ? 0.2 * sm / (n * n) : 0.0;
    for (int ip = 0; ip < n - 1; ++ip)
      for (int iq = ip + 1; iq < n; ++iq) {
        double g = 100. * std::fabs(a[ip][iq]);
        if (it > 4 && std::fabs(d[ip]) + g == std::fabs(d[ip]) && std::fabs(d[iq]) + g == std::fabs(d[iq])) {
          a[ip][iq] = 0.0;
        } else if (std::fabs(a[ip][iq]) > tresh) {
          double h = d[iq] - d[ip], t;
          if (std::fabs(h) + g == std::fabs(h)) {
            t = a[ip][iq] / h;
          } else {
            const double theta = 0.5 * h / a[ip][iq];
            t = 1. / (std::fabs(theta) + std::sqrt(1. + theta * theta));
            if (theta < 0.0) t = -t;
          }
          const double c = 1. / std::sqrt(1 + t * t), s = t * c, tau = s / (1. + c);
          h = t * a[ip][iq];
          z[ip] -= h;
          z[iq] += h;
          d[ip] -= h;
          d[iq] += h;
          a[ip][iq] = 0.0;
          for (int j = 0; j < ip; ++j) {
            g = a[j][ip];
            h = a[j][iq];
            a[j][ip] = g - s * (h + g * tau);
            a[j][iq] = h + s * (g - h * tau);
          }
          for (int j = ip + 1; j < iq; ++j) {
            g = a[ip][j];
            h = a[j][iq];
            a[ip][j] = g - s * (h + g * tau);
            a[j][iq] = h + s * (g - h * tau);
          }
          for (int j = iq + 1; j < n; ++j) {
            g = a[ip][j];
            h = a[iq][j];
            a[ip][j] = g - s * (h + g * tau);
            a[iq][j] = h + s * (g - h * tau);
          }
          for (int j = 0; j < n; ++j) {
            g = v[j][ip];
            h = v[j][iq];
            v[j][ip] = g - s * (h + g * tau);
            v[j][iq] = h + s * (g - h * tau);
          }
        }
      }
    for (int ip = 0; ip < n; ++ip) {
      b[ip] = b[ip] + z[ip];
      d[ip] = b[ip];
      z[ip] = 0.0;
    }
  }
}

}  // namespace

template <class T>
void antisym_t(const T u[3], T uu[3][3]) {
  uu[2][0] = -u[1];
  uu[2][1] = u[0];
  uu[0][1] = -u[2];
  uu[1][0] = -uu[0][1];
  uu[1][2] = -uu[2][1];
  uu[0][2] = -uu[2][0];
  uu[0][0] = uu[1][1] = uu[2][2] = T(0.0);
}

// best/difco.f:104-401 from the four raw friction blocks (Ktt, Ktr, Krt, Krr, as summed in
// difco.f:53-103): the centre of resistance, the diffusion tensors and the centre of diffusion.  T is
// double, or std::complex<double> for complex-step derivatives.  out as bgpu_best_difco's.
template <class T>
void difco_post(T Ktt[3][3], T Ktr[3][3], T Krt[3][3], T Krr[3][3], double cg, T out[60]) {
  T uu[3][3], aux[3][3];
  uu[0][0] = Ktt[1][1] + Ktt[2][2];
  uu[1][1] = Ktt[0][0] + Ktt[2][2];
  uu[2][2] = Ktt[1][1] + Ktt[0][0];
  uu[0][1] = -Ktt[0][1];
  uu[0][2] = -Ktt[0][2];
  uu[2][1] = -Ktt[1][2];
  uu[1][0] = uu[0][1];
  uu[1][2] = uu[2][1];
  uu[2][0] = uu[0][2];
  Krt[0][2] = (Krt[0][2] + Ktr[2][0]) * 0.5;
  Krt[2][0] = (Krt[2][0] + Ktr[0][2]) * 0.5;
  Krt[0][1] = (Krt[0][1] + Ktr[1][0]) * 0.5;
  Krt[1][0] = (Krt[1][0] + Ktr[0][1]) * 0.5;
  Krt[1][2] = (Krt[1][2] + Ktr[2][1]) * 0.5;
  Krt[2][1] = (Krt[2][1] + Ktr[1][2]) * 0.5;
  Krt[0][0] = (Krt[0][0] + Ktr[0][0]) * 0.5;
  Krt[1][1] = (Krt[1][1] + Ktr[1][1]) * 0.5;
  Krt[2][2] = (Krt[2][2] + Ktr[2][2]) * 0.5;
  T sur1 = -Krt[2][1] + Krt[1][2];
  T sur2 = -Krt[0][2] + Krt[2][0];
  T sur3 = -Krt[1][0] + Krt[0][1];
  matin3_t<T>(uu, aux);
  T urc[3], udr[3];
  for (int j = 0; j < 3; ++j) urc[j] = aux[j][0] * sur1 + aux[j][1] * sur2 + aux[j][2] * sur3;
  antisym_t<T>(urc, uu);
  T Krr2[3][3], Krt2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T temp = 0.0;
      for (int k = 0; k < 3; ++k)
        temp = temp + uu[i][k] * (Ktt[k][0] * uu[0][j] + Ktt[k][1] * uu[1][j] + Ktt[k][2] * uu[2][j]);
      const T temp1 = Krt[0][i] * uu[0][j] + Krt[1][i] * uu[1][j] + Krt[2][i] * uu[2][j];
      const T temp2 = uu[i][0] * Krt[0][j] + uu[i][1] * Krt[1][j] + uu[i][2] * Krt[2][j];
      Krr2[i][j] = Krr[i][j] - temp + temp1 - temp2;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Krt2[i][j] = Krt[i][j] + Ktt[i][0] * uu[0][j] + Ktt[i][1] * uu[1][j] + Ktt[i][2] * uu[2][j];
  T Kttinv[3][3], M[3][3], Drr[3][3], Dtr[3][3], Dtt[3][3];
  matin3_t<T>(Ktt, Kttinv);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T temp = 0.0;
      for (int k = 0; k < 3; ++k)
        temp = temp + Krt2[i][k] * (Kttinv[k][0] * Krt2[j][0] + Kttinv[k][1] * Krt2[j][1] + Kttinv[k][2] * Krt2[j][2]);
      M[i][j] = Krr2[i][j] - temp;
    }
  matin3_t<T>(M, Drr);
  if (cg == 0)
    for (auto& r : Drr)
      for (T& v : r) v = 4.0 * v / 3.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T temp = 0.0;
      for (int k = 0; k < 3; ++k)
        temp = temp + Kttinv[i][k] * (Krt2[0][k] * Drr[0][j] + Krt2[1][k] * Drr[1][j] + Krt2[2][k] * Drr[2][j]);
      Dtr[i][j] = -temp;
      if (cg == 0) Dtr[i][j] = 4.0 * Dtr[i][j] / 3.0;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T temp = 0.0;
      for (int k = 0; k < 3; ++k)
        temp = temp + Kttinv[i][k] * (Krt2[0][k] * Dtr[j][0] + Krt2[1][k] * Dtr[j][1] + Krt2[2][k] * Dtr[j][2]);
      Dtt[i][j] = Kttinv[i][j] - temp;
      if (cg == 0) Dtt[i][j] = 4.0 * Dtt[i][j] / 3.0;
    }
  uu[0][0] = Drr[1][1] + Drr[2][2];
  uu[1][1] = Drr[0][0] + Drr[2][2];
  uu[2][2] = Drr[1][1] + Drr[0][0];
  uu[0][1] = -Drr[0][1];
  uu[0][2] = -Drr[0][2];
  uu[2][1] = -Drr[2][1];
  uu[1][0] = uu[0][1];
  uu[1][2] = uu[2][1];
  uu[2][0] = uu[0][2];
  sur1 = Dtr[2][1] - Dtr[1][2];
  sur2 = Dtr[0][2] - Dtr[2][0];
  sur3 = Dtr[1][0] - Dtr[0][1];
  matin3_t<T>(uu, aux);
  for (int j = 0; j < 3; ++j) udr[j] = aux[j][0] * sur1 + aux[j][1] * sur2 + aux[j][2] * sur3;
  antisym_t<T>(udr, uu);
  T Dtt2[3][3], Dtr2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T temp = 0.0;
      for (int k = 0; k < 3; ++k)
        temp = temp + uu[i][k] * Drr[k][0] * uu[0][j] + uu[i][k] * Drr[k][1] * uu[1][j] + uu[i][k] * Drr[k][2] * uu[2][j];
      const T temp1 = Dtr[i][0] * uu[0][j] + Dtr[i][1] * uu[1][j] + Dtr[i][2] * uu[2][j];
      const T temp2 = -uu[i][0] * Dtr[j][0] - uu[i][1] * Dtr[j][1] - uu[i][2] * Dtr[j][2];
      Dtt2[i][j] = Dtt[i][j] - temp + temp1 + temp2;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Dtr2[i][j] = Dtr[i][j] - uu[i][0] * Drr[0][j] - uu[i][1] * Drr[1][j] - uu[i][2] * Drr[2][j];
  auto put = [&](int off, const T m[3][3]) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[off + 3 * i + j] = m[i][j];
  };
  put(0, Dtt2);
  put(9, Dtr2);
  put(18, Drr);
  for (int j = 0; j < 3; ++j) {
    out[27 + j] = urc[j];
    out[30 + j] = udr[j];
  }
  put(33, Ktt);
  put(42, Krt2);
  put(51, Krr2);
}

namespace bgpu {

// The derivatives of BEST's D_t and D_r (best/output.f:96-130: TUNIT and RUNIT times a third of
// the traces of Dtt and Drr; the sum of the Jacobi eigenvalues is the trace) with respect to the four
// raw friction blocks K[0..3] = Ktt, Ktr, Krt, Krr (row-major [j][i], as summed in
// best/difco.f:53-103), by complex-step differentiation of difco_post: exact to rounding, since
// the tensors are analytic in K (matin3 pivots on the real parts).
void difco_post_gradient(const double K[4][9], double cg, double dDt[4][9], double dDr[4][9]) {
  const double temperature = 293.15, eta = 0.01002, pi = 3.141592653;
  const double tunit = (1.38066E-16) * temperature * 1.0E8 / (8.0 * eta * pi);
  const double runit = tunit * 1.0e16;
  double scale = 0.0;
  for (int b = 0; b < 4; ++b)
    for (int e = 0; e < 9; ++e) scale = std::max(scale, std::fabs(K[b][e]));
  const double h = 1e-20 * (scale > 0.0 ? scale : 1.0);
  using C = std::complex<double>;
  for (int b = 0; b < 4; ++b)
    for (int e = 0; e < 9; ++e) {
      C Kc[4][3][3];
      for (int bb = 0; bb < 4; ++bb)
        for (int ee = 0; ee < 9; ++ee) Kc[bb][ee / 3][ee % 3] = C(K[bb][ee], (bb == b && ee == e) ? h : 0.0);
      C out[60];
      difco_post<C>(Kc[0], Kc[1], Kc[2], Kc[3], cg, out);
      dDt[b][e] = tunit * (out[0].imag() + out[4].imag() + out[8].imag()) / 3.0 / h;
      dDr[b][e] = runit * (out[18].imag() + out[22].imag() + out[26].imag()) / 3.0 / h;
    }
}

}  // namespace bgpu

extern "C" {

int bgpu_best_setup(int n, const double* tri, int iarea, double truearea, double* v1, double* v2, double* v3,
                    double* area, double* afac, double* totarea, double* centroid, int* icomp, int* ncomp, int* nopen,
                    int* ndef) {
  if (n < 1) return 1;
  setup_arrays(n, tri, iarea, truearea, v1, v2, v3, area, afac, totarea, centroid);
  compon(n, v1, v2, v3, icomp, ncomp, nopen);
  // best.f:324-337
  *ndef = 1;
  if (*nopen > 0) {
    for (int t = 0; t < n; ++t) icomp[t] = 1;
  } else if (*ncomp > 1) {
    *ndef = *ncomp;
  }
  return 0;
}

int bgpu_best_deflation(int n, const double* v1, const double* v2, const double* v3, const double* area, int ndef,
                        const int* icomp, double diagm, double* xmu, double* gdef) {
  double xmu2 = 0.0;
  for (int t = 0; t < n; ++t) {
    const double v21x = v2[t] - v1[t], v21y = v2[n + t] - v1[n + t], v21z = v2[2 * (size_t)n + t] - v1[2 * (size_t)n + t];
    const double v31x = v3[t] - v1[t], v31y = v3[n + t] - v1[n + t], v31z = v3[2 * (size_t)n + t] - v1[2 * (size_t)n + t];
    const double xnx = v31y * v21z - v31z * v21y, xny = v31z * v21x - v31x * v21z, xnz = v31x * v21y - v31y * v21x;
    const double xnl = std::sqrt(xnx * xnx + xny * xny + xnz * xnz);
    xmu[3 * (size_t)t] = area[t] * xnx / xnl;
    xmu[3 * (size_t)t + 1] = area[t] * xny / xnl;
    xmu[3 * (size_t)t + 2] = area[t] * xnz / xnl;
    xmu2 = xmu2 + xmu[3 * (size_t)t] * xmu[3 * (size_t)t] + xmu[3 * (size_t)t + 1] * xmu[3 * (size_t)t + 1] +
           xmu[3 * (size_t)t + 2] * xmu[3 * (size_t)t + 2];
  }
  if (ndef <= 1) {
    gdef[0] = diagm / xmu2;
    return 0;
  }
  for (int k = 0; k < ndef; ++k) gdef[k] = 0.0;
  for (int t = 0; t < n; ++t) {
    const int k = icomp[t] - 1;
    gdef[k] = gdef[k] + xmu[3 * (size_t)t] * xmu[3 * (size_t)t] + xmu[3 * (size_t)t + 1] * xmu[3 * (size_t)t + 1] +
              xmu[3 * (size_t)t + 2] * xmu[3 * (size_t)t + 2];
  }
  for (int k = 0; k < ndef; ++k) gdef[k] = diagm / gdef[k];
  return 0;
}

void bgpu_best_rhs6(int n, const double* x, double* b) {
  const size_t n3 = 3 * (size_t)n;
  std::fill(b, b + 6 * n3, 0.0);
  for (int t = 0; t < n; ++t) {
    const size_t i0 = 3 * (size_t)t;
    const double X = x[t], Y = x[n + t], Z = x[2 * (size_t)n + t];
    b[i0 + 0] = 1.0;
    b[n3 + i0 + 1] = 1.0;
    b[2 * n3 + i0 + 2] = 1.0;
    b[3 * n3 + i0 + 1] = -Z;
    b[3 * n3 + i0 + 2] = Y;
    b[4 * n3 + i0 + 0] = Z;
    b[4 * n3 + i0 + 2] = -X;
    b[5 * n3 + i0 + 0] = -Y;
    b[5 * n3 + i0 + 1] = X;
  }
}

void bgpu_best_strain5(int n, const double* x, double* v) {
  const size_t n3 = 3 * (size_t)n;
  std::fill(v, v + 5 * n3, 0.0);
  for (int t = 0; t < n; ++t) {
    const size_t i0 = 3 * (size_t)t;
    const double X = x[t], Y = x[n + t], Z = x[2 * (size_t)n + t];
    v[i0 + 0] = 0.5 * Y;
    v[i0 + 1] = 0.5 * X;
    v[n3 + i0 + 0] = 0.5 * Z;
    v[n3 + i0 + 2] = 0.5 * X;
    v[2 * n3 + i0 + 1] = 0.5 * Z;
    v[2 * n3 + i0 + 2] = 0.5 * Y;
    v[3 * n3 + i0 + 0] = 0.5 * X;
    v[3 * n3 + i0 + 1] = -0.5 * Y;
    v[4 * n3 + i0 + 0] = 0.5 * X;
    v[4 * n3 + i0 + 2] = -0.5 * Z;
  }
}

// out: Dtt[9] Dtr[9] Drr[9] urc[3] udr[3] Ktt[9] KrtCR[9] KrrCR[9], each 3x3 row-major (out[3i+j] = M(i+1,j+1))
int bgpu_best_difco(int n, const double* x, const double* area, double cg, const double* b6, double* out) {
  const size_t n3 = 3 * (size_t)n;
  Mat3 Ktt{}, Ktr{}, Krt{}, Krr{};
  for (int mx = 0; mx < 6; ++mx) {
    const double* B = b6 + (size_t)mx * n3;
    double fto[3] = {0, 0, 0}, tto[3] = {0, 0, 0};
    for (int t = 0; t < n; ++t) {
      const double F1 = B[3 * (size_t)t], F2 = B[3 * (size_t)t + 1], F3 = B[3 * (size_t)t + 2];
      const double X = x[t], Y = x[n + t], Z = x[2 * (size_t)n + t];
      const double T1 = Y * F3 - Z * F2, T2 = Z * F1 - X * F3, T3 = X * F2 - Y * F1;
      fto[0] = fto[0] - area[t] * F1;
      fto[1] = fto[1] - area[t] * F2;
      fto[2] = fto[2] - area[t] * F3;
      tto[0] = tto[0] - area[t] * T1;
      tto[1] = tto[1] - area[t] * T2;
      tto[2] = tto[2] - area[t] * T3;
    }
    const double temp = 1.0 / 1.0;
    const int i = mx < 3 ? mx : mx - 3;
    for (int j = 0; j < 3; ++j) {
      if (mx < 3) {
        Ktt[j][i] = -fto[j] * temp;
        Ktr[j][i] = -tto[j] * temp;
      } else {
        Krt[j][i] = -fto[j] * temp;
        Krr[j][i] = -tto[j] * temp;
      }
    }
  }
  difco_post<double>(Ktt, Ktr, Krt, Krr, cg, out);
  return 0;
}

// best/visco.f:24-213; v5: the 5 strain-flow solutions, b6: DIFCO's solutions (unit translations in
// columns 0-2).  out: chiprime, d1, d2, d3.
int bgpu_best_visco(int n, const double* x_in, const double* area, double cg, int icov, const double* v5_in,
                    const double* b6, double* out) {
  const size_t n3 = 3 * (size_t)n;
  std::vector<double> X(x_in, x_in + n3), V0(v5_in, v5_in + 5 * n3);
  double d1 = 0, d2 = 0, d3 = 0;
  auto V = [&](int l, size_t i) -> double& { return V0[(size_t)l * n3 + i]; };
  if (icov) {
    // H(N,L,K,M) from the unit-translation solutions, G(N,L,K) = 2 V0 (visco.f:36-61)
    double BB[3][3] = {}, C1 = 0, C2 = 0, C3 = 0;
    for (int t = 0; t < n; ++t) {
      double G[5][3], H[5][3][3];
      for (int k = 0; k < 3; ++k) {
        for (int l = 0; l < 5; ++l) G[l][k] = 2.0 * V(l, 3 * (size_t)t + k);
        const double E1 = b6[3 * (size_t)t + k], E2 = b6[n3 + 3 * (size_t)t + k], E3 = b6[2 * n3 + 3 * (size_t)t + k];
        H[0][k][0] = E2; H[0][k][1] = E1; H[0][k][2] = 0.0;
        H[1][k][0] = E3; H[1][k][1] = 0.0; H[1][k][2] = E1;
        H[2][k][0] = 0.0; H[2][k][1] = E3; H[2][k][2] = E2;
        H[3][k][0] = E1; H[3][k][1] = -E2; H[3][k][2] = 0.0;
        H[4][k][0] = E1; H[4][k][1] = 0.0; H[4][k][2] = -E3;
      }
      auto h = [&](int l, int k, int m) { return H[l - 1][k - 1][m - 1]; };
      auto g = [&](int l, int k) { return G[l - 1][k - 1]; };
      const double A = area[t], x1 = X[t], x2 = X[n + t], x3 = X[2 * (size_t)n + t];
      BB[0][0] = BB[0][0] + A * (3 * (h(1, 2, 1) + h(2, 3, 1)) + 2 * (h(4, 1, 1) + h(5, 1, 1)));
      BB[0][1] = BB[0][1] + A * (-4 * h(4, 2, 1) + 3 * (h(1, 1, 1) + h(1, 2, 2) + h(2, 3, 2) + h(3, 3, 1)) +
                                 2 * (h(4, 1, 2) + h(5, 1, 2) + h(5, 2, 1)));
      BB[0][2] = BB[0][2] + A * (-4 * h(5, 3, 1) + 3 * (h(1, 2, 3) + h(2, 1, 1) + h(2, 3, 3) + h(3, 2, 1)) +
                                 2 * (h(4, 1, 3) + h(4, 3, 1) + h(5, 1, 3)));
      BB[1][1] = BB[1][1] + A * (-4 * h(4, 2, 2) + 3 * (h(1, 1, 2) + h(3, 3, 2)) + 2 * h(5, 2, 2));
      BB[1][2] = BB[1][2] + A * (-4 * h(4, 2, 3) + 3 * (h(3, 2, 2) + h(3, 3, 3) + h(1, 1, 3) + h(2, 1, 2)) +
                                 2 * (h(4, 3, 2) + h(5, 2, 3)));
      BB[2][2] = BB[2][2] + A * (-4 * h(5, 3, 3) + 3 * (h(2, 1, 3) + h(3, 2, 3)) + 2 * h(4, 3, 3));
      C1 = C1 + A * (-3 * g(1, 2) - 3 * g(2, 3) - 2 * g(4, 1) - 2 * g(5, 1) -
                     x1 * (3 * (h(1, 2, 1) + h(2, 3, 1)) + 2 * (h(4, 1, 1) + h(5, 1, 1))) -
                     x2 * (3 * (h(1, 1, 1) + h(3, 3, 1)) - 4 * h(4, 2, 1) + 2 * h(5, 2, 1)) -
                     x3 * (3 * (h(2, 1, 1) + h(3, 2, 1)) - 4 * h(5, 3, 1) + 2 * h(4, 3, 1)));
      C2 = C2 + A * (-3 * g(1, 1) - 3 * g(3, 3) + 4 * g(4, 2) - 2 * g(5, 2) -
                     x1 * (3 * (h(1, 2, 2) + h(2, 3, 2)) + 2 * (h(4, 1, 2) + h(5, 1, 2))) -
                     x2 * (3 * (h(1, 1, 2) + h(3, 3, 2)) - 4 * h(4, 2, 2) + 2 * h(5, 2, 2)) -
                     x3 * (3 * (h(2, 1, 2) + h(3, 2, 2)) - 4 * h(5, 3, 2) + 2 * h(4, 3, 2)));
      C3 = C3 + A * (-3 * g(2, 1) - 3 * g(3, 2) - 2 * g(4, 3) + 4 * g(5, 3) -
                     x1 * (3 * (h(1, 2, 3) + h(2, 3, 3)) + 2 * (h(4, 1, 3) + h(5, 1, 3))) -
                     x2 * (3 * (h(1, 1, 3) + h(3, 3, 3)) - 4 * h(4, 2, 3) + 2 * h(5, 2, 3)) -
                     x3 * (3 * (h(2, 1, 3) + h(3, 2, 3)) - 4 * h(5, 3, 3) + 2 * h(4, 3, 3)));
    }
    BB[0][0] = BB[0][0] / 15.;
    BB[0][1] = BB[0][1] / 30.;
    BB[0][2] = BB[0][2] / 30.;
    BB[1][0] = BB[0][1];
    BB[1][1] = BB[1][1] / 15.;
    BB[1][2] = BB[1][2] / 30.;
    BB[2][0] = BB[0][2];
    BB[2][1] = BB[1][2];
    BB[2][2] = BB[2][2] / 15.;
    C1 = C1 / 30.;
    C2 = C2 / 30.;
    C3 = C3 / 30.;
    Mat3 BBI;
    matin3(BB, BBI);
    d1 = BBI[0][0] * C1 + BBI[0][1] * C2 + BBI[0][2] * C3;
    d2 = BBI[1][0] * C1 + BBI[1][1] * C2 + BBI[1][2] * C3;
    d3 = BBI[2][0] * C1 + BBI[2][1] * C2 + BBI[2][2] * C3;
    for (int t = 0; t < n; ++t) {
      X[t] = X[t] - d1;
      X[n + t] = X[n + t] - d2;
      X[2 * (size_t)n + t] = X[2 * (size_t)n + t] - d3;
    }
    for (size_t i = 0; i < n3; ++i) {
      const double E1 = b6[i], E2 = b6[n3 + i], E3 = b6[2 * n3 + i];
      V(0, i) = V(0, i) - 0.5 * (d2 * E1 + d1 * E2);
      V(1, i) = V(1, i) - 0.5 * (d3 * E1 + d1 * E3);
      V(2, i) = V(2, i) - 0.5 * (d3 * E2 + d2 * E3);
      V(3, i) = V(3, i) - 0.5 * (d1 * E1 - d2 * E2);
      V(4, i) = V(4, i) - 0.5 * (d1 * E1 - d3 * E3);
    }
  }
  double c112 = 0, c213 = 0, c323 = 0, c411 = 0, c422 = 0, c433 = 0, c511 = 0, c522 = 0, c533 = 0;
  for (int t = 0; t < n; ++t) {
    const size_t i0 = 3 * (size_t)t;
    const double A = area[t], x1 = X[t], x2 = X[n + t], x3 = X[2 * (size_t)n + t];
    c112 = c112 + A * (V(0, i0) * x2 + V(0, i0 + 1) * x1);
    c213 = c213 + A * (V(1, i0) * x3 + V(1, i0 + 2) * x1);
    c323 = c323 + A * (V(2, i0 + 1) * x3 + V(2, i0 + 2) * x2);
    c411 = c411 + A * V(3, i0) * x1;
    c422 = c422 + A * V(3, i0 + 1) * x2;
    c433 = c433 + A * V(3, i0 + 2) * x3;
    c511 = c511 + A * V(4, i0) * x1;
    c522 = c522 + A * V(4, i0 + 1) * x2;
    c533 = c533 + A * V(4, i0 + 2) * x3;
  }
  c112 = 0.5 * c112;
  c213 = 0.5 * c213;
  c323 = 0.5 * c323;
  const double pi = 3.1415926535897932385;
  double chip = 8 * pi * (0.2 * (c112 + c213 + c323) + (c411 - 2 * c422 + c433 + c511 + c522 - 2 * c533) / 15.0);
  if (cg == 0) chip = 0.75 * chip;
  out[0] = chip;
  out[1] = d1;
  out[2] = d2;
  out[3] = d3;
  return 0;
}

// best/output.f:96-130: eigenvalue traces and the cgs values.  tensors as bgpu_best_difco's out.
// out: [0] 1/3 Tr Dtt (1/A), [1] 1/3 Tr Drr (1/A^3), [2] DTRANS (cm^2/s), [3] DR (1/s)
void bgpu_best_traces(const double* tensors, double* out) {
  const double temperature = 293.15, eta = 0.01002, pi = 3.141592653;
  const double tunit = (1.38066E-16) * temperature * 1.0E8 / (8.0 * eta * pi);
  const double runit = tunit * 1.0e16;
  Mat3 Dtt, Drr;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      Dtt[i][j] = tensors[3 * i + j];
      Drr[i][j] = tensors[18 + 3 * i + j];
    }
  double dr[3], dt[3];
  jacobi3(Drr, dr);
  jacobi3(Dtt, dt);
  out[1] = (dr[0] + dr[1] + dr[2]) / 3.;
  out[0] = (dt[0] + dt[1] + dt[2]) / 3.;
  out[2] = tunit * out[0];
  out[3] = runit * out[1];
}


// Least squares of y against 1/N (the reference gives no formula beyond "extrapolated linearly in
// 1/N", README.md:12-16): centred sums, so that the intercept is not the difference of large terms.
double bgpu_best_extrapolate(int count, const int* n, const double* y, double* slope) {
  if (count < 2) {
    if (slope) *slope = 0.0;
    return count == 1 ? y[0] : 0.0;
  }
  double mx = 0.0, my = 0.0;
  for (int i = 0; i < count; ++i) {
    mx += 1.0 / n[i];
    my += y[i];
  }
  mx /= count;
  my /= count;
  double sxx = 0.0, sxy = 0.0;
  for (int i = 0; i < count; ++i) {
    const double dx = 1.0 / n[i] - mx;
    sxx += dx * dx;
    sxy += dx * (y[i] - my);
  }
  const double b = sxx > 0.0 ? sxy / sxx : 0.0;
  if (slope) *slope = b;
  return my - b * mx;
}

}  // extern "C"

namespace {

// Fortran Ew.d (0.ddddE+xx), right-justified in w characters.
std::string fmtE(double v, int w, int d) {
  char buf[64];
  if (v == 0.0) {
    std::snprintf(buf, sizeof buf, "0.%0*dE+00", d, 0);
  } else {
    int e = (int)std::floor(std::log10(std::fabs(v))) + 1;
    double m = std::fabs(v) / std::pow(10.0, e);
    char mb[32];
    std::snprintf(mb, sizeof mb, "%.*f", d, m);
    if (mb[0] == '1') {  // rounding carried to 1.000
      e += 1;
      std::snprintf(mb, sizeof mb, "%.*f", d, std::fabs(v) / std::pow(10.0, e));
    }
    std::snprintf(buf, sizeof buf, "%s%s%s%02d", v < 0 ? "-" : "", mb, e < 0 ? "E-" : "E+", std::abs(e));
  }
  std::string s(buf);
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

std::string line3(const double* m, int row) {
  return "   " + fmtE(m[3 * row], 12, 5) + "   " + fmtE(m[3 * row + 1], 12, 5) + "   " + fmtE(m[3 * row + 2], 12, 5);
}

void drain_log(FILE* lg) {
  char buf[1024];
  for (;;) {
    const int k = bhm_log_line(buf, 1023);
    if (k < 0) break;
    buf[k] = 0;
    if (lg) std::fprintf(lg, " %s\n", buf);
  }
}

}  // namespace

extern "C" int bgpu_best_run(const char* infile, int iarea, int cg_zero, int ivisco, int icov, double wm,
                             int precision, double* results) {
  FILE* in = std::fopen(infile, "r");
  if (!in) {
    std::fprintf(stderr, "best_gpu: cannot open %s\n", infile);
    return 1;
  }
  char head[512];
  if (!std::fgets(head, sizeof head, in)) {
    std::fclose(in);
    return 1;
  }
  double hn = 0, truearea = 0, truevol = 0;
  const int nh = std::sscanf(head, "%lf %lf %lf", &hn, &truearea, &truevol);
  const int n = (int)hn;
  if (n < 1 || (iarea && nh < 3)) {
    std::fprintf(stderr, "best_gpu: bad header in %s (need NAR TRUEAREA TRUEVOL with area correction)\n", infile);
    std::fclose(in);
    return 1;
  }
  std::vector<double> tri(9 * (size_t)n);
  for (size_t i = 0; i < tri.size(); ++i)
    if (std::fscanf(in, "%lf", &tri[i]) != 1) {
      std::fprintf(stderr, "best_gpu: %s ends early\n", infile);
      std::fclose(in);
      return 1;
    }
  std::fclose(in);
  // output names as best.f:225-250 builds them
  std::string base(infile);
  if (ivisco) base += "v";
  if (icov) base += "c";
  if (wm > 0) base += "m";
  if (!iarea) base += "n";
  if (cg_zero) base += "p";
  FILE* lg = std::fopen((base + ".log").c_str(), "w");
  const double cg = cg_zero ? 0.0 : 1.0;
  std::vector<double> v1(3 * (size_t)n), v2(3 * (size_t)n), v3(3 * (size_t)n), area(n), x(3 * (size_t)n);
  std::vector<int> icomp(n);
  double afac = 1, totarea = 0, cen[3];
  int ncomp = 0, nopen = 0, ndef = 1;
  bgpu_best_setup(n, tri.data(), iarea, truearea, v1.data(), v2.data(), v3.data(), area.data(), &afac, &totarea, cen,
                  icomp.data(), &ncomp, &nopen, &ndef);
  if (lg) {
    std::fprintf(lg, " BEST (GPU backend) control gtensor value= %g\n total area (A^2) = %.15g\n", cg, totarea);
    std::fprintf(lg, " centroid coords = %.15g %.15g %.15g\n", cen[0], cen[1], cen[2]);
    if (nopen > 0) std::fprintf(lg, " warning: %d edges are not shared by exactly two triangles: the surface is open\n", nopen);
    if (ndef > 1) std::fprintf(lg, " surface: %d separate closed surfaces; the normal field of each is deflated\n", ndef);
  }
  int rc = 0;
  if (precision >= 0) bgpu_set_precision(precision);
  if ((rc = bhm_create(n, v1.data(), v2.data(), v3.data(), area.data(), afac, cg, 0)) != 0) {
    drain_log(lg);
    if (lg) std::fclose(lg);
    return rc;
  }
  bhm_incenters(x.data());
  const double diagm = bhm_diag_mean();
  std::vector<double> xmu(3 * (size_t)n), gdef(std::max(1, ndef));
  bgpu_best_deflation(n, v1.data(), v2.data(), v3.data(), area.data(), ndef, icomp.data(), diagm, xmu.data(),
                      gdef.data());
  if (lg) std::fprintf(lg, " normal-field deflation: mean diagonal of GR = %.15g\n", diagm);
  rc = bhm_build(1e-4, precision == 0 ? 1 : 0, 0.1, ndef, gdef.data(), icomp.data(), xmu.data(), 0, ivisco ? 11 : 6);
  drain_log(lg);
  if (rc != 0) {
    if (lg) std::fclose(lg);
    return rc;
  }
  const size_t n3 = 3 * (size_t)n;
  std::vector<double> b(6 * n3), v5(5 * n3);
  bgpu_best_rhs6(n, x.data(), b.data());
  if ((rc = bhm_solve(6, b.data())) != 0) {
    drain_log(lg);
    if (lg) std::fclose(lg);
    return rc;
  }
  double tens[60], vis[4] = {0, 0, 0, 0}, tr[4];
  bgpu_best_difco(n, x.data(), area.data(), cg, b.data(), tens);
  if (ivisco) {
    bgpu_best_strain5(n, x.data(), v5.data());
    if ((rc = bhm_solve(5, v5.data())) != 0) {
      drain_log(lg);
      if (lg) std::fclose(lg);
      return rc;
    }
    bgpu_best_visco(n, x.data(), area.data(), cg, icov, v5.data(), b.data(), vis);
  }
  drain_log(lg);
  bgpu_best_traces(tens, tr);
  // best.f:486-496: only finite results are written
  for (int i = 0; i < 33; ++i)
    if (!std::isfinite(tens[i])) {
      if (lg) std::fprintf(lg, " error: the diffusion tensors are not finite (NaN or Inf); nothing was written to the .be file\n");
      if (lg) std::fclose(lg);
      return 1;
    }
  const double chi = iarea ? vis[0] / truevol : 0.0, etav = wm > 0 ? vis[0] * 0.602214 / wm : 0.0;
  FILE* be = std::fopen((base + ".be").c_str(), "w");
  if (be) {
    // best/output.f:38-171
    std::fprintf(be, " BEST Ver. 4.0 SFSU/ARAGON (GPU backend)\n\n BE - MACROMOLECULE TRANSPORT TENSORS\n\n");
    std::fprintf(be, "     Area (A^2)            %s\n", fmtE(totarea, 12, 5).c_str());
    if (iarea) {
      std::fprintf(be, "     True Area (A^2)       %s\n     Areafactor                 %7.4f\n", fmtE(truearea, 12, 5).c_str(), afac);
      std::fprintf(be, "     True Volume (A^3)     %s\n", fmtE(truevol, 12, 5).c_str());
    }
    if (wm > 0) std::fprintf(be, "     Molecular Weight (g/mol)  %8.1f\n", wm);
    std::fprintf(be, "     Temperature (K)            %8.3f\n     Solvent Viscosity (Poise)  %8.5f\n", 293.15, 0.01002);
    std::fprintf(be, "     Number of Surface Patches    %5d\n\n", n);
    if (cg_zero) std::fprintf(be, "  PRE-AVERAGING USED FOR THIS CALCULATION\n");
    std::fprintf(be, "\n  Centroid Coordinates (A)\n   %s   %s   %s\n", fmtE(cen[0], 12, 5).c_str(), fmtE(cen[1], 12, 5).c_str(), fmtE(cen[2], 12, 5).c_str());
    std::fprintf(be, "  Vector between Center of Resistance/Centroid \n%s\n", line3(tens + 27, 0).c_str());
    std::fprintf(be, "  Vector between Centers of Diffusion/Resistance\n%s\n", line3(tens + 30, 0).c_str());
    std::fprintf(be, "\n  Diffusion Tensors in Center of Mobility\n\n  Dtt Tensor (1/A)\n");
    for (int r = 0; r < 3; ++r) std::fprintf(be, "%s\n", line3(tens, r).c_str());
    std::fprintf(be, "\n  Symmetric Dtr Tensor (1/A^2)\n");
    for (int r = 0; r < 3; ++r) std::fprintf(be, "%s\n", line3(tens + 9, r).c_str());
    std::fprintf(be, "\n   Drr TENSOR (1/A^3)\n");
    for (int r = 0; r < 3; ++r) std::fprintf(be, "%s\n", line3(tens + 18, r).c_str());
    std::fprintf(be, "\n  1/3 Trace DRR(EXACT) =%s 1/s\n\n", fmtE(tr[3], 15, 5).c_str());
    std::fprintf(be, "  1/3 Trace DTT(EXACT) =%s cm^2/s\n\n", fmtE(tr[2], 15, 5).c_str());
    if (ivisco) {
      if (icov) std::fprintf(be, " %s AT THE CENTER OF VISCOSITY\n  Vector between Center of Viscosity/Centroid\n     Dx = %s  Dy = %s  Dz = %s\n",
                             wm > 0 ? "INTRINSIC VISCOSITY" : "VISCOSITY FACTOR", fmtE(vis[1], 12, 5).c_str(), fmtE(vis[2], 12, 5).c_str(), fmtE(vis[3], 12, 5).c_str());
      else std::fprintf(be, " %s AT THE CENTROID\n", wm > 0 ? "INTRINSIC VISCOSITY" : "VISCOSITY FACTOR");
      if (iarea) std::fprintf(be, "\n     CHI               %s\n", fmtE(chi, 16, 6).c_str());
      std::fprintf(be, "     CHI*VOLUME (A^3)  %s\n\n", fmtE(vis[0], 16, 6).c_str());
      if (wm > 0) std::fprintf(be, "     ETA (cm^3/g)      %s\n\n", fmtE(etav, 16, 6).c_str());
    }
    std::fclose(be);
  }
  if (lg) std::fclose(lg);
  if (results) {
    std::memcpy(results, tens, 60 * sizeof(double));
    results[60] = vis[0];
    results[61] = vis[1];
    results[62] = vis[2];
    results[63] = vis[3];
    results[64] = tr[2];
    results[65] = tr[3];
    results[66] = chi;
    results[67] = etav;
  }
  bhm_destroy();
  return 0;
}
