// FP64 field solve of one run in ONE launch: a cluster of kFieldCtas CTAs
// on as many SMs computes the 2D real-to-complex DFT of rho, the spectral
// Poisson solve and the three inverse transforms (phi, Ex, Ey), exchanging
// rows and columns through distributed shared memory.
//
// Reference: Efield::solve_poisson_fftw (miniapps/vlp4d/thrust/efield.cpp:
// 43-105, with the filter of efield.cpp:27-33) on FFTW/cuFFT plans
// (lib/Cuda_FFT.hpp:83-183): a D2Z transform of rho - 1 (cases 10, 20,
// field.cpp:65-72), the mode-wise solve, a Z2D transform of each of phi_hat,
// ex_hat, ey_hat.  The mode-wise solve is the function k_poisson_solve runs
// (poisson_mode, field.cu), so both paths share its arithmetic; the
// transforms differ from cuFFT's only in rounding.
//
// Decomposition (cluster rank c of C CTAs, R = ny / C rows each, the
// half-spectrum columns kx = c, c + C, ... <= nx/2 each):
//   1. rows iy in [cR, cR + R): complex DFT along x of (rho - offset, 0);
//   -- cluster barrier --
//   2. own columns: gather the rows' values of column kx from every CTA
//      (distributed shared memory), DFT along y: rho_hat;
//   3. the mode-wise solve: phi_hat, ex_hat, ey_hat of the own columns;
//   4. inverse DFT along y of the three spectra;
//   -- cluster barrier --
//   5. own rows, per field: gather the row's half spectrum from the column
//      owners, extend it by Hermitian symmetry, inverse DFT along x, real
//      part to global memory (rho <- phi, ex, ey);
//   -- cluster barrier (no CTA leaves while another reads its memory) --
// Lines of power-of-two length use radix-4 Stockham passes (self-sorting,
// one CTA barrier per pass over all lines of a phase; a radix-2 pass last
// for odd powers); other lengths a direct DFT.  Twiddles exp(2 pi i m / n) from sincospi.  All waits are the
// hardware's CTA and cluster barriers, which every thread of every CTA
// reaches the same number of times.
#include <cstdlib>
#include <cstring>

#include "internal.cuh"
#include "poisson.cuh"

namespace vlp4d {

namespace {

// Cluster sizes: 8 (portable) or 16 (non-portable, where the device allows it).
constexpr int kFieldThreads = 512;
constexpr int kFieldMaxN = 128;    // largest nx, ny of the cluster solve

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// The value at `local` (a shared-memory address of this CTA's layout) in
// the shared memory of cluster CTA `rank`.
__device__ __forceinline__ double2 ld_cluster(const double2 *local, unsigned rank) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(local);
  unsigned ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  double2 v;
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(ra) : "memory");
  return v;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// DFT of `lines` contiguous lines of length n (line l at buf + l * n):
// out[k] = sum_j in[j] w^(jk), w = exp(sign 2 pi i / n), tw[m] = exp(2 pi i
// m / n) (conjugated for sign < 0).  The result is in buf or tmp (returned);
// both hold lines * n values.  Ends with a CTA barrier.
__device__ double2 *line_dft(double2 *buf, double2 *tmp, int lines, int n, const double2 *tw, bool inverse) {
  const double sgn = inverse ? 1. : -1.;
  if ((n & (n - 1)) == 0) {
    const int ln = __ffs(n) - 1;  // log2(n)
    double2 *x = buf, *y = tmp;
    int ls = 0;  // log2 of the length of the sub-transforms done so far
    // Radix-4 passes: out[d + p*ns] = sum_m (x[j + m n/4] w^(m k)) i^(sgn m p),
    // j in [0, n/4), k = j mod ns, d = (j / ns) * 4 ns + k, w = exp(sgn 2 pi
    // i / (4 ns)).
    for (; ls + 2 <= ln; ls += 2) {
      const int ns = 1 << ls, lq = ln - 2, quarter = 1 << lq;
      const int tshift = ln - ls - 2;  // w^(m k) = tw[(m k) << tshift]
      for (int b = threadIdx.x; b < lines << lq; b += blockDim.x) {
        const int l = b >> lq, j = b & (quarter - 1);
        const int k = j & (ns - 1);
        const int base = l * n;
        double2 a0 = x[base + j], a1 = x[base + j + quarter], a2 = x[base + j + 2 * quarter],
                a3 = x[base + j + 3 * quarter];
        if (k) {
          const double2 t1 = tw[k << tshift], t2 = tw[(2 * k) << tshift], t3 = tw[(3 * k) << tshift];
          a1 = cmul(a1, make_double2(t1.x, sgn * t1.y));
          a2 = cmul(a2, make_double2(t2.x, sgn * t2.y));
          a3 = cmul(a3, make_double2(t3.x, sgn * t3.y));
        }
        const double2 s02 = make_double2(a0.x + a2.x, a0.y + a2.y), d02 = make_double2(a0.x - a2.x, a0.y - a2.y);
        const double2 s13 = make_double2(a1.x + a3.x, a1.y + a3.y), d13 = make_double2(a1.x - a3.x, a1.y - a3.y);
        // (sgn i) * d13
        const double2 r13 = make_double2(-sgn * d13.y, sgn * d13.x);
        const int d = base + ((j >> ls) << (ls + 2)) + k;
        y[d] = make_double2(s02.x + s13.x, s02.y + s13.y);
        y[d + ns] = make_double2(d02.x + r13.x, d02.y + r13.y);
        y[d + 2 * ns] = make_double2(s02.x - s13.x, s02.y - s13.y);
        y[d + 3 * ns] = make_double2(d02.x - r13.x, d02.y - r13.y);
      }
      __syncthreads();
      double2 *s = x;
      x = y;
      y = s;
    }
    // A last radix-2 pass when log2(n) is odd.
    if (ls < ln) {
      const int ns = 1 << ls, lh = ln - 1, half = 1 << lh;
      for (int b = threadIdx.x; b < lines << lh; b += blockDim.x) {
        const int l = b >> lh, j = b & (half - 1);
        const int k = j & (ns - 1);
        const int base = l * n;
        const double2 v0 = x[base + j];
        const double2 t = tw[k];  // k * n / (2 ns) = k (ns = n / 2)
        const double2 v1 = cmul(x[base + j + half], make_double2(t.x, sgn * t.y));
        const int d = base + ((j >> ls) << (ls + 1)) + k;
        y[d] = make_double2(v0.x + v1.x, v0.y + v1.y);
        y[d + ns] = make_double2(v0.x - v1.x, v0.y - v1.y);
      }
      __syncthreads();
      double2 *s = x;
      x = y;
      y = s;
    }
    return x;
  }
  for (int o = threadIdx.x; o < lines * n; o += blockDim.x) {
    const int l = o / n, k = o - l * n;
    const double2 *xl = buf + (size_t)l * n;
    double sr = 0., si = 0.;
    int m = 0;
    for (int j = 0; j < n; ++j) {
      const double2 v = xl[j], t = tw[m];
      const double wi = sgn * t.y;
      sr += v.x * t.x - v.y * wi;
      si += v.x * wi + v.y * t.x;
      m += k;
      if (m >= n) m -= n;
    }
    tmp[o] = make_double2(sr, si);
  }
  __syncthreads();
  return tmp;
}

struct FieldArgs {
  double *rho;       // in: rho (nx*ny); out: phi.  ex, ey at rho + fstride, + 2 fstride
  long long fstride;
  int nx, ny;
  double offset;     // subtracted from rho before the transform (1 for cases 10, 20, else 0)
  double kx0, ky0, normcoeff;
};

// Shared memory: two row buffers (R x nx), two column buffers (3 spectra x
// Kc columns x ny), the x and y twiddles.
struct FieldSmem {
  int R, Kc;
  size_t rows_elems, cols_elems;
  __host__ __device__ FieldSmem(int nx, int ny, int ctas) {
    R = ny / ctas;
    Kc = (nx / 2 + 1 + ctas - 1) / ctas;
    rows_elems = (size_t)R * nx;
    cols_elems = (size_t)3 * Kc * ny;
  }
  // The forward solve: two row buffers of three fields' rows each (the
  // inverse x transforms of phi, Ex, Ey run as one batch), two column
  // buffers, the twiddles.
  __host__ __device__ size_t bytes(int nx, int ny) const {
    return sizeof(double2) * (6 * rows_elems + 2 * cols_elems + nx + ny);
  }
};

template <int kFieldCtas>
__global__ void __launch_bounds__(kFieldThreads) k_field_cluster(FieldArgs a) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const int nx = a.nx, ny = a.ny, nxh = nx / 2 + 1;
  const FieldSmem L(nx, ny, kFieldCtas);
  const int R = L.R, Kc = L.Kc;
  double2 *rowA = reinterpret_cast<double2 *>(fsm);
  double2 *rowB = rowA + 3 * L.rows_elems;
  double2 *colA = rowB + 3 * L.rows_elems;
  double2 *colB = colA + L.cols_elems;
  double2 *twx = colB + L.cols_elems;
  double2 *twy = twx + nx;
  const unsigned c = cluster_rank();
  for (int m = threadIdx.x; m < nx; m += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / nx, &sn, &cs);
    twx[m] = make_double2(cs, sn);
  }
  for (int m = threadIdx.x; m < ny; m += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / ny, &sn, &cs);
    twy[m] = make_double2(cs, sn);
  }
  // 1. Own rows along x.
  const int iy0 = (int)c * R;
  for (int i = threadIdx.x; i < R * nx; i += blockDim.x)
    rowA[i] = make_double2(a.rho[(size_t)iy0 * nx + i] - a.offset, 0.);
  __syncthreads();
  const double2 *rows = line_dft(rowA, rowB, R, nx, twx, false);
  cluster_barrier();
  // 2. Own columns along y: column q is kx = c + q * C (Kc slots; the last
  // ones of some CTAs are past nx/2 and stay unused).
  int nq = 0;
  for (int kx = (int)c; kx < nxh; kx += kFieldCtas) ++nq;
  for (int i = threadIdx.x; i < nq * ny; i += blockDim.x) {
    const int q = i / ny, iy = i - q * ny;
    const int kx = (int)c + q * kFieldCtas;
    colA[i] = ld_cluster(rows + (size_t)(iy % R) * nx + kx, (unsigned)(iy / R));
  }
  __syncthreads();
  const double2 *rhat = line_dft(colA, colB, nq, ny, twy, false);
  // 3. The mode-wise solve into the other column buffer: spectra
  // phi_hat, ex_hat, ey_hat at slots [0, Kc), [Kc, 2Kc), [2Kc, 3Kc).
  double2 *spec = rhat == colA ? colB : colA;
  double2 *spare = rhat == colA ? colA : colB;
  for (int i = threadIdx.x; i < nq * ny; i += blockDim.x) {
    const int q = i / ny, iy = i - q * ny;
    const int kx = (int)c + q * kFieldCtas;
    double2 e1, e2, r1;
    poisson_mode(kx, iy, ny, rhat[i], a.kx0, a.ky0, a.normcoeff, e1, e2, r1);
    spec[(size_t)q * ny + iy] = r1;
    spec[(size_t)(Kc + q) * ny + iy] = e1;
    spec[(size_t)(2 * Kc + q) * ny + iy] = e2;
  }
  __syncthreads();
  // 4. Inverse along y of the 3 Kc column slots (the unused ones too: the
  // slots are contiguous; their values are never read).
  const double2 *cols = line_dft(spec, spare, 3 * Kc, ny, twy, true);
  cluster_barrier();
  // 5. Own rows of the three fields (line f * R + r): half spectra from the
  // column owners, Hermitian extension, inverse along x, real part.
  for (int i = threadIdx.x; i < 3 * R * nxh; i += blockDim.x) {
    const int l = i / nxh, kx = i - l * nxh;
    const int f = l / R, r = l - f * R;
    const int owner = kx % kFieldCtas, q = kx / kFieldCtas;
    rowA[(size_t)l * nx + kx] = ld_cluster(cols + (size_t)(f * Kc + q) * ny + iy0 + r, (unsigned)owner);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * R * (nx - nxh); i += blockDim.x) {
    const int l = i / (nx - nxh), kx = nxh + (i - l * (nx - nxh));
    const double2 v = rowA[(size_t)l * nx + (nx - kx)];
    rowA[(size_t)l * nx + kx] = make_double2(v.x, -v.y);
  }
  __syncthreads();
  const double2 *out = line_dft(rowA, rowB, 3 * R, nx, twx, true);
  for (int i = threadIdx.x; i < 3 * R * nx; i += blockDim.x) {
    const int f = i / (R * nx), e = i - f * (R * nx);
    a.rho[f * a.fstride + (size_t)iy0 * nx + e] = out[i].x;
  }
  cluster_barrier();
}


// The transpose of the field solve (the reverse mode's lam_rho = D^T (gex,
// gey)), with the same decomposition: rows of gex and gey along x; --
// cluster barrier --; own columns of both along y, the mode-wise
// lam_hat = (conj(hx_hat) gx_hat + conj(hy_hat) gy_hat) / (nx*ny) with the
// impulse-response spectra hx_hat, hy_hat (half-spectrum layout of the
// forward D2Z, ky * (nx/2+1) + kx), the inverse along y; -- cluster barrier
// --; own rows of lam_hat: Hermitian extension, inverse along x, real part
// into lam_rho; -- cluster barrier --.
struct FieldTArgs {
  const double *gex, *gey;
  const double2 *hx, *hy;
  double *lam;
  int nx, ny;
  double norm;
};

// Shared memory of k_field_cluster_t: four row buffers (gex and gey rows
// and their pass partners), four column buffers, the twiddles.
__host__ __device__ inline size_t field_t_bytes(int nx, int ny, int ctas) {
  const FieldSmem L(nx, ny, ctas);
  return sizeof(double2) * (4 * L.rows_elems + 4 * (size_t)L.Kc * ny + nx + ny);
}

template <int kFieldCtas>
__global__ void __launch_bounds__(kFieldThreads) k_field_cluster_t(FieldTArgs a) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const int nx = a.nx, ny = a.ny, nxh = nx / 2 + 1;
  const FieldSmem L(nx, ny, kFieldCtas);
  const int R = L.R, Kc = L.Kc;
  const size_t ce = (size_t)Kc * ny;
  double2 *rx = reinterpret_cast<double2 *>(fsm);
  double2 *rxt = rx + L.rows_elems;
  double2 *ry = rxt + L.rows_elems;
  double2 *ryt = ry + L.rows_elems;
  double2 *cx = ryt + L.rows_elems;
  double2 *cxt = cx + ce;
  double2 *cy = cxt + ce;
  double2 *cyt = cy + ce;
  double2 *twx = cyt + ce;
  double2 *twy = twx + nx;
  const unsigned c = cluster_rank();
  for (int m = threadIdx.x; m < nx; m += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / nx, &sn, &cs);
    twx[m] = make_double2(cs, sn);
  }
  for (int m = threadIdx.x; m < ny; m += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / ny, &sn, &cs);
    twy[m] = make_double2(cs, sn);
  }
  const int iy0 = (int)c * R;
  for (int i = threadIdx.x; i < R * nx; i += blockDim.x) {
    rx[i] = make_double2(a.gex[(size_t)iy0 * nx + i], 0.);
    ry[i] = make_double2(a.gey[(size_t)iy0 * nx + i], 0.);
  }
  __syncthreads();
  const double2 *rowsx = line_dft(rx, rxt, R, nx, twx, false);
  const double2 *rowsy = line_dft(ry, ryt, R, nx, twx, false);
  cluster_barrier();
  int nq = 0;
  for (int kx = (int)c; kx < nxh; kx += kFieldCtas) ++nq;
  for (int i = threadIdx.x; i < nq * ny; i += blockDim.x) {
    const int q = i / ny, iy = i - q * ny;
    const int kx = (int)c + q * kFieldCtas;
    const size_t off = (size_t)(iy % R) * nx + kx;
    const unsigned owner = (unsigned)(iy / R);
    cx[i] = ld_cluster(rowsx + off, owner);
    cy[i] = ld_cluster(rowsy + off, owner);
  }
  __syncthreads();
  const double2 *gxh = line_dft(cx, cxt, nq, ny, twy, false);
  const double2 *gyh = line_dft(cy, cyt, nq, ny, twy, false);
  // lam_hat of the own columns into a buffer neither spectrum occupies.
  double2 *lam = gxh == cx ? cxt : cx;
  double2 *lamt = gyh == cy ? cyt : cy;
  for (int i = threadIdx.x; i < nq * ny; i += blockDim.x) {
    const int q = i / ny, iy = i - q * ny;
    const int kx = (int)c + q * kFieldCtas;
    const double2 g1 = gxh[i], g2 = gyh[i];
    const double2 p = a.hx[(size_t)iy * nxh + kx], r = a.hy[(size_t)iy * nxh + kx];
    lam[i] = make_double2((p.x * g1.x + p.y * g1.y + r.x * g2.x + r.y * g2.y) * a.norm,
                          (p.x * g1.y - p.y * g1.x + r.x * g2.y - r.y * g2.x) * a.norm);
  }
  __syncthreads();
  const double2 *cols = line_dft(lam, lamt, nq, ny, twy, true);
  cluster_barrier();
  for (int i = threadIdx.x; i < R * nxh; i += blockDim.x) {
    const int r = i / nxh, kx = i - r * nxh;
    rx[(size_t)r * nx + kx] = ld_cluster(cols + (size_t)(kx / kFieldCtas) * ny + iy0 + r, (unsigned)(kx % kFieldCtas));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < R * (nx - nxh); i += blockDim.x) {
    const int r = i / (nx - nxh), kx = nxh + (i - r * (nx - nxh));
    const double2 v = rx[(size_t)r * nx + (nx - kx)];
    rx[(size_t)r * nx + kx] = make_double2(v.x, -v.y);
  }
  __syncthreads();
  const double2 *out = line_dft(rx, rxt, R, nx, twx, true);
  for (int i = threadIdx.x; i < R * nx; i += blockDim.x) a.lam[(size_t)iy0 * nx + i] = out[i].x;
  cluster_barrier();
}
}  // namespace

namespace {

cudaLaunchConfig_t field_config(int nx, int ny, int ctas, cudaLaunchAttribute *attr, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kFieldThreads);
  cfg.dynamicSmemBytes = FieldSmem(nx, ny, ctas).bytes(nx, ny);
  cfg.stream = s;
  attr->id = cudaLaunchAttributeClusterDimension;
  attr->val.clusterDim.x = ctas;
  attr->val.clusterDim.y = 1;
  attr->val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int C>
bool cluster_fits(int nx, int ny) {
  if (ny % C) return false;
  const size_t smem = FieldSmem(nx, ny, C).bytes(nx, ny);
  if (cudaFuncSetAttribute(k_field_cluster<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      (C > 8 && cudaFuncSetAttribute(k_field_cluster<C>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                    cudaSuccess)) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchAttribute attr;
  const cudaLaunchConfig_t cfg = field_config(nx, ny, C, &attr, 0);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, k_field_cluster<C>, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    return false;
  }
  return true;
}

}  // namespace

bool field_cluster_available(vlp4d_ctx *c) {
  if (c->field_cluster >= 0) return c->field_cluster > 0;
  c->field_cluster = 0;
  const char *env = getenv("VLP4D_FIELD");
  if (env && strcmp(env, "cufft") == 0) return false;
  const int nx = c->g.n[0], ny = c->g.n[1];
  if (nx < 2 || ny < 8 || nx > kFieldMaxN || ny > kFieldMaxN) return false;
  const int want = env && strcmp(env, "cluster8") == 0 ? 8 : 16;
  if (want == 16 && cluster_fits<16>(nx, ny)) c->field_cluster = 16;
  else if (cluster_fits<8>(nx, ny)) c->field_cluster = 8;
  return c->field_cluster > 0;
}

// The transposed solve on the cluster size the forward solve uses; false
// (cuFFT path) if it does not fit.
bool field_cluster_t_available(vlp4d_ctx *c) {
  if (!field_cluster_available(c)) return false;
  if (c->field_cluster_t >= 0) return c->field_cluster_t > 0;
  c->field_cluster_t = 0;
  const int nx = c->g.n[0], ny = c->g.n[1], C = c->field_cluster;
  const size_t smem = field_t_bytes(nx, ny, C);
  cudaError_t e = C == 16 ? cudaFuncSetAttribute(k_field_cluster_t<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                          : cudaFuncSetAttribute(k_field_cluster_t<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && C == 16)
    e = cudaFuncSetAttribute(k_field_cluster_t<16>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchAttribute attr;
  cudaLaunchConfig_t cfg = field_config(nx, ny, C, &attr, 0);
  cfg.dynamicSmemBytes = smem;
  int clusters = 0;
  e = C == 16 ? cudaOccupancyMaxActiveClusters(&clusters, k_field_cluster_t<16>, &cfg)
              : cudaOccupancyMaxActiveClusters(&clusters, k_field_cluster_t<8>, &cfg);
  if (e != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    return false;
  }
  c->field_cluster_t = 1;
  return true;
}

int launch_field_transpose_cluster(vlp4d_ctx *c, const double *gex, const double *gey, const void *hx_hat,
                                   const void *hy_hat, double *lam_rho, cudaStream_t s) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  FieldTArgs a;
  a.gex = gex;
  a.gey = gey;
  a.hx = static_cast<const double2 *>(hx_hat);
  a.hy = static_cast<const double2 *>(hy_hat);
  a.lam = lam_rho;
  a.nx = nx;
  a.ny = ny;
  a.norm = 1.0 / ((double)nx * ny);
  cudaLaunchAttribute attr;
  cudaLaunchConfig_t cfg = field_config(nx, ny, c->field_cluster, &attr, s);
  cfg.dynamicSmemBytes = field_t_bytes(nx, ny, c->field_cluster);
  if (c->field_cluster == 16) VLP4D_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_field_cluster_t<16>, a));
  else VLP4D_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_field_cluster_t<8>, a));
  return VLP4D_OK;
}

int launch_field_cluster(vlp4d_ctx *c, double offset, cudaStream_t s) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  FieldArgs a;
  a.rho = c->rho;
  a.fstride = (long long)c->fstride;
  a.nx = nx;
  a.ny = ny;
  a.offset = offset;
  a.kx0 = 2 * M_PI / c->g.maxp[0];  // efield.cpp:44-45: 2*pi / maxPhy
  a.ky0 = 2 * M_PI / c->g.maxp[1];
  a.normcoeff = 1.0 / (double)(nx * ny);
  cudaLaunchAttribute attr;
  const cudaLaunchConfig_t cfg = field_config(nx, ny, c->field_cluster, &attr, s);
  if (c->field_cluster == 16) VLP4D_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_field_cluster<16>, a));
  else VLP4D_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_field_cluster<8>, a));
  return VLP4D_OK;
}

}  // namespace vlp4d
