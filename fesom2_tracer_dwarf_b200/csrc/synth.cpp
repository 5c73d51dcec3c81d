// Seeded synthetic inputs for the large analytic configurations: bathymetry,
// a discretely consistent layered flow, and tracer fields.  All arithmetic is
// host FP64; the generator is deterministic for a given seed.
#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <random>

#include "mesh.hpp"

namespace fesom {

template <typename T>
HugeArray<T>::HugeArray(size_t n) : n_(n) {
  if (n == 0) return;
  const size_t huge = size_t(2) << 20;
  bytes_ = (n * sizeof(T) + huge - 1) / huge * huge;
  void *p = mmap(nullptr, bytes_, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  if (p == MAP_FAILED) throw std::bad_alloc();
  madvise(p, bytes_, MADV_HUGEPAGE);  // advisory: 4 KB pages if refused
  p_ = static_cast<T *>(p);
}

template <typename T>
HugeArray<T>::~HugeArray() {
  if (p_) munmap(p_, bytes_);
}

template class HugeArray<double>;
template class HugeArray<int>;

namespace {

struct Rng {
  std::mt19937_64 g;
  explicit Rng(uint64_t s) : g(s) {}
  double uni() { return (double)(g() >> 11) * 0x1.0p-53; }  // [0, 1)
  double normal() {
    double u1 = uni(), u2 = uni();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPiRef * u2);
  }
};

// Smooth field periodic on [0,Lx) x [0,Ly): a few Fourier modes with integer
// wave numbers (so it is continuous across the periodic wrap).
struct Modes {
  int kx[6], ky[6];
  double amp[6], ph[6];
  void draw(Rng &r) {
    for (int q = 0; q < 6; q++) {
      kx[q] = 1 + (int)(r.g() % 4);
      ky[q] = 1 + (int)(r.g() % 4);
      amp[q] = 0.5 + r.uni();
      ph[q] = 2.0 * kPiRef * r.uni();
    }
  }
  double eval(double x, double y, double Lx, double Ly) const {
    double s = 0.0;
    for (int q = 0; q < 6; q++) s += amp[q] * std::sin(2.0 * kPiRef * (kx[q] * x / Lx + ky[q] * y / Ly) + ph[q]);
    return s;
  }
};

}  // namespace

std::vector<int> synth_bathymetry(int nnodes, int nl, uint64_t seed) {
  std::mt19937_64 g(seed);
  std::vector<int> K(nnodes);
  const uint64_t span = (uint64_t)(nl - 2);  // values 3..nl
  for (int n = 0; n < nnodes; n++) K[n] = 3 + (int)(g() % span);
  return K;
}

std::vector<int> synth_bathymetry_smooth(int nx, int ny, bool periodic, int nl, double corr_cells, uint64_t seed) {
  // Gaussian random field from random-phase Fourier modes (integer wave
  // numbers, so it is periodic), mapped through the normal CDF to a uniform
  // marginal on [3, nl]
  Rng r(seed);
  const int nm = 48;
  std::vector<double> kx(nm), ky(nm), ph(nm);
  const double kmax = std::max(1.0, (double)std::max(nx, ny) / std::max(1.0, corr_cells));
  for (int q = 0; q < nm; q++) {
    double a, b;
    do {
      a = std::floor((2.0 * r.uni() - 1.0) * (kmax + 1.0));
      b = std::floor((2.0 * r.uni() - 1.0) * (kmax + 1.0));
    } while (a == 0.0 && b == 0.0);
    kx[q] = a; ky[q] = b;
    ph[q] = 2.0 * kPiRef * r.uni();
  }
  const int ni = periodic ? nx - 1 : nx, nj = periodic ? ny - 1 : ny;
  std::vector<int> K((size_t)ni * nj);
  const double norm = std::sqrt(2.0 / nm);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) {
      const double x = (double)i / (double)(nx - 1), y = (double)j / (double)(ny - 1);
      double g = 0.0;
      for (int q = 0; q < nm; q++) g += std::cos(2.0 * kPiRef * (kx[q] * x + ky[q] * y) + ph[q]);
      g *= norm;                                            // ~ N(0, 1)
      const double u = 0.5 * std::erfc(-g / std::sqrt(2.0));  // ~ U(0, 1)
      int k = 3 + (int)(u * (double)(nl - 2));
      K[(size_t)j * ni + i] = std::min(nl, std::max(3, k));
    }
  return K;
}

void synth_velocity(const MeshHost &m, uint64_t seed, double umax, double mode1_frac, double mode2_frac,
                    double baro_frac, double *uv, double *W) {
  const int N = m.nod2D, T = m.elem2D, E = m.edge2D, nl = m.nl, L = nl - 1;
  Rng rng(seed);
  std::vector<double> xm(N), ym(N);
  for (int n = 0; n < N; n++) { xm[n] = m.coord[2 * n] * kREarth; ym[n] = m.coord[2 * n + 1] * kREarth; }
  // two smooth horizontal patterns per element: U1 = curl(psi1),
  // U2 = curl(psi2) + grad(chi)
  Modes p1, p2, chi, p0;
  p1.draw(rng);
  p2.draw(rng);
  chi.draw(rng);
  if (baro_frac != 0.0) p0.draw(rng);
  std::vector<double> f1(N), f2(N), f3(N);
  for (int n = 0; n < N; n++) {
    f1[n] = p1.eval(xm[n], ym[n], m.Lx, m.Ly);
    f2[n] = p2.eval(xm[n], ym[n], m.Lx, m.Ly);
    f3[n] = chi.eval(xm[n], ym[n], m.Lx, m.Ly);
  }
  const size_t nuv = (size_t)2 * L * T;
  std::memset(uv, 0, nuv * sizeof(double));
  // barotropic part curl(psi0): psi0 zeroed at nodes touching an element dry
  // at the level and on walls, so that on a mesh whose edges all carry
  // edge_tri(1) on their left its edge fluxes sum to zero at every node
  if (baro_frac != 0.0) {
    std::vector<int> shallowest(N, nl);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) shallowest[m.elem_nodes[3 * e + q]] = std::min(shallowest[m.elem_nodes[3 * e + q]], m.nlev_elem[e]);
    std::vector<char> wall(N, 0);
    for (int e = 0; e < E; e++)
      if (m.edge_tri[2 * e + 1] < 0) { wall[m.edge_nodes[2 * e]] = 1; wall[m.edge_nodes[2 * e + 1]] = 1; }
    std::vector<double> f0(N);
    for (int n = 0; n < N; n++) f0[n] = wall[n] ? 0.0 : baro_frac * p0.eval(xm[n], ym[n], m.Lx, m.Ly);
    for (int e = 0; e < T; e++) {
      const int *en = &m.elem_nodes[3 * e];
      const double *gs = &m.grad_sca[6 * e];
      for (int k = 0; k < m.nlev_elem[e] - 1; k++) {
        double psi[3];
        for (int q = 0; q < 3; q++) psi[q] = (k + 1) > shallowest[en[q]] - 1 ? 0.0 : f0[en[q]];
        uv[2 * ((size_t)e * L + k)] += -(gs[3] * psi[0] + gs[4] * psi[1] + gs[5] * psi[2]);
        uv[2 * ((size_t)e * L + k) + 1] += gs[0] * psi[0] + gs[1] * psi[1] + gs[2] * psi[2];
      }
    }
  }
  std::vector<double> c1(L), c2(L);
  for (int e = 0; e < T; e++) {
    const int *en = &m.elem_nodes[3 * e];
    const double *gs = &m.grad_sca[6 * e];
    auto gx = [&](const std::vector<double> &f) { return gs[0] * f[en[0]] + gs[1] * f[en[1]] + gs[2] * f[en[2]]; };
    auto gy = [&](const std::vector<double> &f) { return gs[3] * f[en[0]] + gs[4] * f[en[1]] + gs[5] * f[en[2]]; };
    const double u1 = -gy(f1), v1 = gx(f1);
    const double u2 = -gy(f2) + gx(f3), v2 = gx(f2) + gy(f3);
    // vertical modes with zero thickness-weighted mean over the element's
    // own water column (helem), so the column integral of every edge flux
    // vanishes on uniform and on stretched level sets alike
    const int M = m.nlev_elem[e] - 1;
    const double *h = &m.helem[(size_t)e * L];
    double s1 = 0.0, s2 = 0.0, hs = 0.0;
    for (int k = 0; k < M; k++) {
      c1[k] = std::cos(kPiRef * ((double)k + 0.5) / (double)M);
      c2[k] = std::cos(2.0 * kPiRef * ((double)k + 0.5) / (double)M);
      s1 += c1[k] * h[k];
      s2 += c2[k] * h[k];
      hs += h[k];
    }
    s1 /= hs;
    s2 /= hs;
    for (int k = 0; k < M; k++) {
      const double a1 = mode1_frac * (c1[k] - s1), a2 = mode2_frac * (c2[k] - s2);
      uv[2 * ((size_t)e * L + k)] += a1 * u1 + a2 * u2;
      uv[2 * ((size_t)e * L + k) + 1] += a1 * v1 + a2 * v2;
    }
  }
  double vmax = 0.0;
  for (size_t i = 0; i < nuv / 2; i++) vmax = std::max(vmax, std::hypot(uv[2 * i], uv[2 * i + 1]));
  // umax < 0: -umax is the amplitude itself (same flow on any resolution)
  const double scale = umax < 0.0 ? -umax : (vmax > 0.0 ? umax / vmax : 0.0);
  for (size_t i = 0; i < nuv; i++) uv[i] *= scale;

  // horizontal divergence D(n,k) of the edge volume fluxes, with the same
  // segment rule the advection kernels use
  HugeArray<double> D((size_t)L * N);
  for (int e = 0; e < E; e++) {
    const int n1 = m.edge_nodes[2 * e], n2 = m.edge_nodes[2 * e + 1];
    const int t1 = m.edge_tri[2 * e], t2 = m.edge_tri[2 * e + 1];
    const int nl1 = m.nlev_elem[t1] - 1, nl2 = t2 >= 0 ? m.nlev_elem[t2] - 1 : 0;
    const double *c = &m.edge_cross[4 * e];
    for (int k = 0; k < std::max(nl1, nl2); k++) {
      double v = 0.0;
      if (k < nl1) v += (-uv[2 * ((size_t)t1 * L + k) + 1] * c[0] + uv[2 * ((size_t)t1 * L + k)] * c[1]) * m.helem[(size_t)t1 * L + k];
      if (k < nl2) v += (uv[2 * ((size_t)t2 * L + k) + 1] * c[2] - uv[2 * ((size_t)t2 * L + k)] * c[3]) * m.helem[(size_t)t2 * L + k];
      D[(size_t)n1 * L + k] += v;
      D[(size_t)n2 * L + k] -= v;
    }
  }
  // W from bottom to top: W(k) A(k) = W(k+1) A(k+1) - D(k); W = 0 at the
  // bottom and at the surface
  std::memset(W, 0, (size_t)nl * N * sizeof(double));
  for (int n = 0; n < N; n++) {
    const int nlev = m.nlev_node[n];
    for (int i = nlev - 1; i >= 2; i--) {  // 1-based interface i, top of layer i
      const double Ai = m.area[(size_t)n * nl + i - 1], Ai1 = m.area[(size_t)n * nl + i];
      const double flux_below = W[(size_t)n * nl + i] * Ai1;
      W[(size_t)n * nl + i - 1] = Ai > 0.0 ? (flux_below - D[(size_t)n * L + i - 1]) / Ai : 0.0;
    }
    W[(size_t)n * nl + 0] = 0.0;
  }
}

void synth_tracer(const MeshHost &m, uint64_t seed, int kind, double *T) {
  const int N = m.nod2D, L = m.nl - 1;
  Rng r(seed);
  std::memset(T, 0, (size_t)L * N * sizeof(double));
  if (kind == 0) {
    double bx[8], by[8], bs[8], ba[8];
    for (int b = 0; b < 8; b++) {
      bx[b] = r.uni() * m.Lx; by[b] = r.uni() * m.Ly;
      bs[b] = (0.03 + 0.07 * r.uni()) * m.Lx; ba[b] = 5.0 + 10.0 * r.uni();
    }
    for (int n = 0; n < N; n++) {
      const double x = m.coord[2 * n] * kREarth, y = m.coord[2 * n + 1] * kREarth;
      double blob = 0.0;
      for (int b = 0; b < 8; b++) {
        double dx = std::fabs(x - bx[b]), dy = std::fabs(y - by[b]);
        if (m.periodic) { dx = std::min(dx, m.Lx - dx); dy = std::min(dy, m.Ly - dy); }
        blob += ba[b] * std::exp(-(dx * dx + dy * dy) / (bs[b] * bs[b]));
      }
      for (int k = 0; k < m.nlev_node[n] - 1; k++) T[(size_t)n * L + k] = 20.0 * r.uni() + blob;
    }
  } else if (kind == 1) {
    for (int n = 0; n < N; n++)
      for (int k = 0; k < m.nlev_node[n] - 1; k++) T[(size_t)n * L + k] = 35.0 + 0.5 * r.normal();
  } else {
    // smooth, resolution-independent: Gaussian blobs plus periodic tanh fronts,
    // weakly varying with depth
    double bx[6], by[6], bs[6], ba[6], fk[3][2], fp[3], fa[3];
    for (int b = 0; b < 6; b++) {
      bx[b] = r.uni() * m.Lx; by[b] = r.uni() * m.Ly;
      bs[b] = (0.04 + 0.06 * r.uni()) * m.Lx; ba[b] = (r.uni() < 0.5 ? -1.0 : 1.0) * (3.0 + 5.0 * r.uni());
    }
    for (int f = 0; f < 3; f++) {
      fk[f][0] = (double)(1 + (int)(r.g() % 3)) * (r.uni() < 0.5 ? -1.0 : 1.0);
      fk[f][1] = (double)(1 + (int)(r.g() % 3));
      fp[f] = 2.0 * kPiRef * r.uni(); fa[f] = 1.0 + 2.0 * r.uni();
    }
    const double H = m.zbar[0] - m.zbar[m.nl - 1];
    for (int n = 0; n < N; n++) {
      const double x = m.coord[2 * n] * kREarth, y = m.coord[2 * n + 1] * kREarth;
      double v = 15.0;
      for (int b = 0; b < 6; b++) {
        double dx = std::fabs(x - bx[b]), dy = std::fabs(y - by[b]);
        if (m.periodic) { dx = std::min(dx, m.Lx - dx); dy = std::min(dy, m.Ly - dy); }
        v += ba[b] * std::exp(-(dx * dx + dy * dy) / (bs[b] * bs[b]));
      }
      for (int f = 0; f < 3; f++)
        v += fa[f] * std::tanh(4.0 * std::sin(2.0 * kPiRef * (fk[f][0] * x / m.Lx + fk[f][1] * y / m.Ly) + fp[f]));
      for (int k = 0; k < m.nlev_node[n] - 1; k++) {
        const double z = 0.5 * (m.zbar[k] + m.zbar[k + 1]);
        T[(size_t)n * L + k] = v * (1.0 - 0.2 * (m.zbar[0] - z) / H);
      }
    }
  }
}

void analytic_driver_fields(const MeshHost &m, std::vector<double> &T, std::vector<double> &S,
                            std::vector<double> &uv, std::vector<double> &W) {
  const int N = m.nod2D, nz = m.nl - 1;
  const double Lx = m.Lx, Ly = m.Ly, xc = 0.5 * Lx, yc = 0.5 * Ly;
  T.assign((size_t)nz * N, 0.0);
  S.assign((size_t)nz * N, 0.0);
  for (int n = 0; n < N; n++) {
    const double xn = m.coord[2 * n] * kREarth, yn = m.coord[2 * n + 1] * kREarth;
    const double r = std::sqrt((xn - xc) * (xn - xc) + (yn - yc) * (yn - yc));
    for (int k = 1; k <= nz; k++) {
      const double zn = (double)(k - 1) / (double)(nz - 1);
      T[(size_t)n * nz + k - 1] = 15.0 + 5.0 * std::sin(2.0 * kPiRef * xn / Lx) * std::cos(2.0 * kPiRef * yn / Ly) - 10.0 * zn;
      S[(size_t)n * nz + k - 1] = 34.0 + 2.0 * std::exp(-(r * r) / ((0.1 * Lx) * (0.1 * Lx))) * (1.0 - zn);
    }
  }
  uv.assign((size_t)2 * nz * m.elem2D, 0.0);
  for (size_t i = 0; i < (size_t)nz * m.elem2D; i++) uv[2 * i] = 0.1;
  W.assign((size_t)m.nl * N, 0.0);
}

}  // namespace fesom
