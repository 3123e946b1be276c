// ocfd_aux.cu -- hybrid shock sensor, device mesh/metric initialisation,
// filtering and the diagnostic reductions.
//
// Reductions (sensor-2 mean, show_flow_msg, ana_box) use a fixed grid and a
// fixed-order two-level tree, so they are bitwise reproducible run to run; the
// reference's sequential sums round differently (within a few ulp).
#include "ocfd_kernels.h"
#include "ocfd_schemes.cuh"

namespace ocfd {

constexpr int RED_BLOCKS = 148 * 4;
constexpr int RED_THREADS = 256;

size_t reduce_scratch_doubles(const Grid& g) { return (size_t)RED_BLOCKS * 16 + 64; }

// fixed-order block sum of NV values; thread 0 gets the result
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sm) {
  for (int q = 0; q < NV; q++) sm[q * RED_THREADS + threadIdx.x] = v[q];
  __syncthreads();
  for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int q = 0; q < NV; q++) sm[q * RED_THREADS + threadIdx.x] += sm[q * RED_THREADS + threadIdx.x + s];
    __syncthreads();
  }
  for (int q = 0; q < NV; q++) v[q] = sm[q * RED_THREADS];
}

template <int NV>
__global__ void k_final_sum(const double* part, int nb, double* out) {
  __shared__ double sm[NV * RED_THREADS];
  double v[NV];
  for (int q = 0; q < NV; q++) v[q] = 0.0;
  for (int b = threadIdx.x; b < nb; b += RED_THREADS)
    for (int q = 0; q < NV; q++) v[q] += part[b * NV + q];
  block_sum<NV>(v, sm);
  if (threadIdx.x == 0)
    for (int q = 0; q < NV; q++) out[q] = v[q];
}

// central derivative of a haloed FP64 array (OCFD_dx0/dy0/dz0)
__device__ __forceinline__ double d0h_bnd(const double* q, long long s, int l, int nn, int cd8, const DCoef& c, int dir) {
  auto at = [&](int off) -> double { return q[off * s]; };
  const double h = c.h[dir], a1 = c.a1[dir], a2 = c.a2[dir], a3 = c.a3[dir];
  double r = 0.0;
  if (l == 1) r = (-3.0 * at(0) + 4.0 * at(1) - at(2)) / (2.0 * h);
  else if (l == 2) r = (at(1) - at(-1)) / (2.0 * h);
  else if (l == 3) r = (8.0 * (at(1) - at(-1)) - (at(2) - at(-2))) / (12.0 * h);
  else if (cd8 && l == 4) r = a1 * (at(3) - at(-3)) + a2 * (at(2) - at(-2)) + a3 * (at(1) - at(-1));
  if (l == nn) r = (at(-2) - 4.0 * at(-1) + 3.0 * at(0)) / (2.0 * h);
  else if (l == nn - 1) r = (at(1) - at(-1)) / (2.0 * h);
  else if (l == nn - 2) r = (8.0 * (at(1) - at(-1)) - (at(2) - at(-2))) / (12.0 * h);
  else if (cd8 && l == nn - 3) r = a1 * (at(3) - at(-3)) + a2 * (at(2) - at(-2)) + a3 * (at(1) - at(-1));
  return r;
}
__device__ __forceinline__ double d0h(const double* q, long long s, int l, int nn, int periodic, int cd8,
                                      const DCoef& c, int dir) {
  const int lo = cd8 ? 4 : 3, hi = cd8 ? nn - 3 : nn - 2;
  if (periodic || (l > lo && l < hi)) {
    if (!cd8) return c.a1[dir] * (q[3 * s] - q[-3 * s]) + c.a2[dir] * (q[2 * s] - q[-2 * s]) + c.a3[dir] * (q[s] - q[-s]);
    return c.c1[dir] * (q[s] - q[-s]) + c.c2[dir] * (q[2 * s] - q[-2 * s]) + c.c3[dir] * (q[3 * s] - q[-3 * s]) +
           c.c4[dir] * (q[4 * s] - q[-4 * s]);
  }
  return d0h_bnd(q, s, l, nn, cd8, c, dir);
}

__device__ __forceinline__ void decode(const Grid& G, long long t, int& i, int& j, int& k) {
  i = (int)(t % G.nx) + 1;
  j = (int)((t / G.nx) % G.ny) + 1;
  k = (int)(t / ((long long)G.nx * G.ny)) + 1;
}

// ---------------------------------------------------------------------------
// comput_Rhybrid (OCFD_SetHybrid.f90:17-152)
struct Patches {
  int n;
  int box[16][6];
};

// one thread a point, 32 x 8 points of a plane a block (no index decoding)
__global__ void __launch_bounds__(256) k_rh_sensor1(Grid G, double p00, const double* d, const double* T,
                                                    double* rh) {
  {
    const int i = blockIdx.x * 32 + (threadIdx.x & 31) + 1;
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5) + 1;
    const int k = blockIdx.z + 1;
    if (i > G.nx || j > G.ny) return;
    const long long c = G.ih(i, j, k);
    auto P = [&](long long h) -> double { return p00 * d[h] * T[h]; };
    double r = 0.0;
    const long long s[3] = {1, (long long)G.nxh, (long long)G.nxh * G.nyh};
    const double pc = P(c);
    double acc;
    {
      const double pm = P(c - s[0]), pp = P(c + s[0]);
      acc = fabs((pm - 2.0 * pc + pp) / (pm + 2.0 * pc + pp));
    }
    {
      const double pm = P(c - s[1]), pp = P(c + s[1]);
      acc = acc + fabs((pm - 2.0 * pc + pp) / (pm + 2.0 * pc + pp));
    }
    {
      const double pm = P(c - s[2]), pp = P(c + s[2]);
      r = acc + fabs((pm - 2.0 * pc + pp) / (pm + 2.0 * pc + pp));
    }
    rh[c] = r;
  }
}

__global__ void k_rh_p(long long nh, double p00, const double* d, const double* T, double* p) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nh; t += (long long)gridDim.x * blockDim.x)
    p[t] = p00 * d[t] * T[t];
}

__global__ void __launch_bounds__(RED_THREADS) k_rh_sensor2(Grid G, Phys ph, DCoef dc, const double* p,
                                                            const double* Akx, const double* Aky, const double* Akz,
                                                            const double* Aix, const double* Aiy, const double* Aiz,
                                                            const double* Asx, const double* Asy, const double* Asz,
                                                            double* rh, double* part) {
  __shared__ double sm[RED_THREADS];
  const int cd8 = ph.scheme_vis == 6;
  double v[1] = {0.0};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    const double pk = d0h(p + c, 1, i, G.nx, ph.periodic[0], cd8, dc, 0);
    const double pi = d0h(p + c, G.nxh, j, G.ny, ph.periodic[1], cd8, dc, 1);
    const double ps = d0h(p + c, (long long)G.nxh * G.nyh, k, G.nz, ph.periodic[2], cd8, dc, 2);
    const double px = pk * Akx[c] + pi * Aix[c] + ps * Asx[c];
    const double py = pk * Aky[c] + pi * Aiy[c] + ps * Asy[c];
    const double pz = pk * Akz[c] + pi * Aiz[c] + ps * Asz[c];
    const double r = sqrt(px * px + py * py + pz * pz);
    rh[c] = r;
    v[0] += r;
  }
  block_sum<1>(v, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void k_rh_scale(Grid G, const double* sum, double* rh) {
  const double dp_av = sum[0] / (1.0 * G.nx * G.ny * G.nz);
  const double dp_av1 = 1.0 / (dp_av + 1.0e-30);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    rh[c] = rh[c] * dp_av1;
  }
}

__global__ void k_rh_patch(Grid G, Patches P, double* rh) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    double r = rh[c];
    for (int m = 0; m < P.n; m++) {
      const int* b = P.box[m];
      if (i >= b[0] && i <= b[1] && j >= b[2] && j <= b[3] && k >= b[4] && k <= b[5]) r = r + 100.0;
    }
    rh[c] = r;
  }
}

size_t rhybrid_scratch_doubles(const Grid& g) { return (size_t)g.nh + RED_BLOCKS + 16; }

cudaError_t launch_rhybrid(const Grid& g, const Phys& ph, const DCoef& dc, const double* d, const double* T,
                           const double* const met[22], double* rh, double* scratch, int sensor,
                           const double* hp, cudaStream_t st) {
  const double p00 = 1.0 / (ph.gamma * ph.ma * ph.ma);
  if (sensor == 1) {
    k_rh_sensor1<<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz), 256, 0, st>>>(g, p00, d, T, rh);
  } else {
    double* p = scratch;
    double* part = scratch + g.nh;
    double* sum = part + RED_BLOCKS;
    k_rh_p<<<148 * 8, 256, 0, st>>>(g.nh, p00, d, T, p);
    k_rh_sensor2<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, ph, dc, p, met[3], met[4], met[5], met[6], met[7], met[8],
                                                     met[9], met[10], met[11], rh, part);
    k_final_sum<1><<<1, RED_THREADS, 0, st>>>(part, RED_BLOCKS, sum);
    k_rh_scale<<<148 * 8, 256, 0, st>>>(g, sum, rh);
  }
  // forced patches (OCFD_SetHybrid.f90:88-110); the reference's :93 assigns
  // Hybrid_para(8) to ie and leaves je undefined -- here both take Hybrid_para(8).
  Patches P;
  P.n = (int)llround(hp[3]);
  if (P.n > 16) P.n = 16;
  if (P.n < 0) P.n = 0;
  for (int m = 0; m < P.n; m++) {
    const double* q = hp + 4 + 6 * m;
    int ib = (int)llround(q[0]), ie = (int)llround(q[3]), jb = (int)llround(q[2]), je = (int)llround(q[3]);
    int kb = (int)llround(q[4]), ke = (int)llround(q[5]);
    P.box[m][0] = ib < 1 ? 1 : ib;
    P.box[m][1] = ie > g.nx ? g.nx : ie;
    P.box[m][2] = jb < 1 ? 1 : jb;
    P.box[m][3] = je > g.ny ? g.ny : je;
    P.box[m][4] = kb < 1 ? 1 : kb;
    P.box[m][5] = ke > g.nz ? g.nz : ke;
  }
  if (P.n > 0) k_rh_patch<<<148 * 8, 256, 0, st>>>(g, P, rh);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// init_mesh (OCFD_mesh.f90:1-58) on the device.
// updata_Axyz_periodic (OCFD_mesh.f90:109-185)
__global__ void k_mesh_shift(Grid G, int px, int py, int pz, double3 si, double3 sj, double3 sk, double* X, double* Y,
                             double* Z) {
  const long long nxl = px ? (long long)LAP * G.ny * G.nz : 0;
  const long long nyl = py ? (long long)LAP * G.nx * G.nz : 0;
  const long long nzl = pz ? (long long)LAP * G.nx * G.ny : 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nxl + nyl + nzl;
       t += (long long)gridDim.x * blockDim.x) {
    long long e = t;
    long long lo, hi;
    double3 s;
    if (e < nxl) {
      const int l = (int)(e % LAP) + 1;
      e /= LAP;
      const int j = (int)(e % G.ny) + 1, k = (int)(e / G.ny) + 1;
      lo = G.ih(1 - l, j, k);
      hi = G.ih(G.nx + l, j, k);
      s = si;
    } else if (e < nxl + nyl) {
      e -= nxl;
      const int i = (int)(e % G.nx) + 1;
      e /= G.nx;
      const int l = (int)(e % LAP) + 1, k = (int)(e / LAP) + 1;
      lo = G.ih(i, 1 - l, k);
      hi = G.ih(i, G.ny + l, k);
      s = sj;
    } else {
      e -= nxl + nyl;
      const int i = (int)(e % G.nx) + 1;
      e /= G.nx;
      const int j = (int)(e % G.ny) + 1, l = (int)(e / G.ny) + 1;
      lo = G.ih(i, j, 1 - l);
      hi = G.ih(i, j, G.nz + l);
      s = sk;
    }
    X[lo] = X[lo] - s.x;
    Y[lo] = Y[lo] - s.y;
    Z[lo] = Z[lo] - s.z;
    X[hi] = X[hi] + s.x;
    Y[hi] = Y[hi] + s.y;
    Z[hi] = Z[hi] + s.z;
  }
}

struct MetPtrs {
  double* m[22];
};

__device__ __forceinline__ void jac_store(double* const* M, long long c, double xi1, double xj1, double xk1, double yi1,
                                          double yj1, double yk1, double zi1, double zj1, double zk1) {
  const double Jac1 = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 -
                             yi1 * xj1 * zk1 - xi1 * zj1 * yk1);
  M[12][c] = Jac1;
  M[3][c] = Jac1 * (yj1 * zk1 - zj1 * yk1);
  M[4][c] = Jac1 * (zj1 * xk1 - xj1 * zk1);
  M[5][c] = Jac1 * (xj1 * yk1 - yj1 * xk1);
  M[6][c] = Jac1 * (yk1 * zi1 - zk1 * yi1);
  M[7][c] = Jac1 * (zk1 * xi1 - xk1 * zi1);
  M[8][c] = Jac1 * (xk1 * yi1 - yk1 * xi1);
  M[9][c] = Jac1 * (yi1 * zj1 - zi1 * yj1);
  M[10][c] = Jac1 * (zi1 * xj1 - xi1 * zj1);
  M[11][c] = Jac1 * (xi1 * yj1 - yi1 * xj1);
}

// comput_Jacobian3d (OCFD_mesh.f90:61-107)
__global__ void k_jacobian(Grid G, Phys ph, DCoef dc, MetPtrs mp) {
  const int cd8 = ph.scheme_vis == 6;
  double* const* M = mp.m;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    const long long s[3] = {1, (long long)G.nxh, (long long)G.nxh * G.nyh};
    const int l[3] = {i, j, k};
    double dd[3][3];  // [x,y,z][i,j,k]
    for (int q = 0; q < 3; q++)
      for (int d = 0; d < 3; d++) dd[q][d] = d0h(M[q] + c, s[d], l[d], G.len(d), ph.periodic[d], cd8, dc, d);
    jac_store(M, c, dd[0][0], dd[0][1], dd[0][2], dd[1][0], dd[1][1], dd[1][2], dd[2][0], dd[2][1], dd[2][2]);
  }
}

// Jac_Ghost_Extent_1st (OCFD_GhostCell.f90:18-160) and the coordinate mirror of
// Jac_Ghost_Extent_2nd (:290-379)
__global__ void k_jac_ghost_coords(Grid G, Phys ph, int order, MetPtrs mp) {
  double* const* M = mp.m;
  long long cnt[6], tot = 0;
  for (int f = 0; f < 6; f++) {
    const int dir = f / 2;
    const long long tr = dir == 0 ? (long long)G.ny * G.nz : (dir == 1 ? (long long)G.nx * G.nz : (long long)G.nx * G.ny);
    cnt[f] = ph.ghost[f] == order ? tr * LAP : 0;
    tot += cnt[f];
  }
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    long long e = t;
    int face = 0;
    while (e >= cnt[face]) e -= cnt[face++];
    const int dir = face / 2, hi = face % 2, nn = G.len(dir);
    const int l = (int)(e % LAP) + 1;
    e /= LAP;
    const int n1 = dir == 0 ? G.ny : G.nx;
    const int a = (int)(e % n1) + 1, b = (int)(e / n1) + 1;
    auto H = [&](int along) -> long long {
      if (dir == 0) return G.ih(along, a, b);
      if (dir == 1) return G.ih(a, along, b);
      return G.ih(a, b, along);
    };
    const int g = hi ? nn + l : 1 - l;
    if (order == 1) {
      const long long hg = H(g), he = H(hi ? nn : 1), he2 = H(hi ? nn - 1 : 2);
      for (int m = 3; m <= 12; m++) M[m][hg] = M[m][he];
      const double fac = hi ? (double)(g - nn) : (1.0 - g);
      for (int m = 0; m < 3; m++) M[m][hg] = M[m][he] + fac * (M[m][he] - M[m][he2]);
    } else {
      const long long hg = H(g), he = H(hi ? nn : 1), hg1 = H(hi ? 2 * nn - g : 2 - g);
      for (int m = 0; m < 3; m++) M[m][hg] = 2.0 * M[m][he] - M[m][hg1];
    }
  }
}

// comput_Jacobian3d_Ghost (OCFD_GhostCell.f90:394-500) for one face
__global__ void k_jac_ghost_metrics(Grid G, Phys ph, int nb, MetPtrs mp) {
  double* const* M = mp.m;
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  int ib, ie, jb, je, kb, ke, ib1, ie1, jb1, je1, kb1, ke1;
  if (nb == 1) { ib = 1 - LAP; ie = 0; jb = 1; je = ny; kb = 1; ke = nz; ib1 = ib; ie1 = 1; jb1 = jb; je1 = je; kb1 = kb; ke1 = ke; }
  else if (nb == 2) { ib = nx + 1; ie = nx + LAP; jb = 1; je = ny; kb = 1; ke = nz; ib1 = nx; ie1 = ie; jb1 = jb; je1 = je; kb1 = kb; ke1 = ke; }
  else if (nb == 3) { ib = 1; ie = nx; jb = 1 - LAP; je = 0; kb = 1; ke = nz; ib1 = ib; ie1 = ie; jb1 = jb; je1 = 1; kb1 = kb; ke1 = ke; }
  else if (nb == 4) { ib = 1; ie = nx; jb = ny + 1; je = ny + LAP; kb = 1; ke = nz; ib1 = ib; ie1 = ie; jb1 = ny; je1 = je; kb1 = kb; ke1 = ke; }
  else if (nb == 5) { ib = 1; ie = nx; jb = 1; je = ny; kb = 1 - LAP; ke = 0; ib1 = ib; ie1 = ie; jb1 = jb; je1 = je; kb1 = kb; ke1 = 1; }
  else { ib = 1; ie = nx; jb = 1; je = ny; kb = nz + 1; ke = nz + LAP; ib1 = ib; ie1 = ie; jb1 = jb; je1 = je; kb1 = nz; ke1 = ke; }
  const long long ni = ie - ib + 1, nj = je - jb + 1, nk = ke - kb + 1;
  const double hh[3] = {ph.hx, ph.hy, ph.hz};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ni * nj * nk; t += (long long)gridDim.x * blockDim.x) {
    const int i = ib + (int)(t % ni), j = jb + (int)((t / ni) % nj), k = kb + (int)(t / (ni * nj));
    const long long c = G.ih(i, j, k);
    const int lc[3] = {i, j, k}, lb1[3] = {ib1, jb1, kb1}, le1[3] = {ie1, je1, ke1};
    double dv[3][3];  // [x,y,z][dir]
    for (int d = 0; d < 3; d++) {
      const long long s = G.hstride(d);
      const double h = hh[d];
      for (int q = 0; q < 3; q++) {
        const double* A = M[q] + c;
        double r;
        if (lc[d] == lb1[d])
          r = (-3.0 * A[0] + 4.0 * A[s] - A[2 * s]) / (2.0 * h);
        else if (lc[d] == le1[d])
          r = (A[-2 * s] - 4.0 * A[-s] + 3.0 * A[0]) / (2.0 * h);
        else if (lc[d] == lb1[d] + 1 || lc[d] == le1[d] - 1)
          r = (A[s] - A[-s]) / (2.0 * h);
        else
          r = (8.0 * (A[s] - A[-s]) - (A[2 * s] - A[-2 * s])) / (12.0 * h);
        dv[q][d] = r;
      }
    }
    jac_store(M, c, dv[0][0], dv[0][1], dv[0][2], dv[1][0], dv[1][1], dv[1][2], dv[2][0], dv[2][1], dv[2][2]);
  }
}

// Jac_Ghost_Userdef (OCFD_GhostCell_UserDef.f90:4-11): mirrored metrics and
// coordinates with the sign of the reflected components flipped -- swept corner
// k- symmetry about z = 0 (Jac_Ghost_Sweptcorner :23-49), flat plate j-
// symmetry about y = 0 (Jac_Ghost_flatplate :76-102).
__global__ void k_jac_ghost_user(Grid G, Phys ph, MetPtrs mp) {
  double* const* M = mp.m;
  const bool sc = ph.ibc == 3 && ph.ghost[4] == -1;
  // Akx Aky Akz Aix Aiy Aiz Asx Asy Asz Ajac (ids 3..12) and Axx Ayy Azz (0..2)
  const int ids[13] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 0, 1, 2};
  const double sgz[13] = {1, 1, -1, 1, 1, -1, -1, -1, 1, 1, 1, 1, -1};
  const double sgy[13] = {1, -1, 1, -1, 1, -1, 1, -1, 1, 1, 1, -1, 1};
  const long long tot = sc ? (long long)G.nx * G.ny * LAP : (long long)G.nx * G.nz * LAP;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    long long h, h1;
    if (sc) {
      const int i = (int)(t % G.nx) + 1, j = (int)((t / G.nx) % G.ny) + 1, k = 1 - LAP + (int)(t / ((long long)G.nx * G.ny));
      h = G.ih(i, j, k);
      h1 = G.ih(i, j, 1 - k);
    } else {
      const int i = (int)(t % G.nx) + 1, k = (int)((t / G.nx) % G.nz) + 1, j = 1 - LAP + (int)(t / ((long long)G.nx * G.nz));
      h = G.ih(i, j, k);
      h1 = G.ih(i, 2 - j, k);
    }
    for (int q = 0; q < 13; q++) {
      const double x = M[ids[q]][h1];
      M[ids[q]][h] = (sc ? sgz[q] : sgy[q]) < 0 ? -x : x;
    }
  }
}

// Akx1 = Akx/Ajac ... over the whole haloed box (OCFD_mesh.f90:41-55)
__global__ void k_metric_div(long long nh, MetPtrs mp) {
  double* const* M = mp.m;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nh; t += (long long)gridDim.x * blockDim.x) {
    const double J = M[12][t];
    for (int m = 0; m < 9; m++) M[13 + m][t] = M[3 + m][t] / J;
  }
}

cudaError_t launch_mesh(const Grid& g, const Phys& ph, const DCoef& dc, double* const met[22],
                        const double span[3][3], bool jac_given, cudaStream_t st) {
  MetPtrs mp;
  for (int m = 0; m < 22; m++) mp.m[m] = met[m];
  PtrList<double> xyz;
  xyz.n = 3;
  for (int q = 0; q < 3; q++) xyz.p[q] = met[q];
  cudaError_t e = launch_halo(g, ph.periodic, xyz, st);
  if (e != cudaSuccess) return e;
  k_mesh_shift<<<148 * 4, 256, 0, st>>>(g, ph.periodic[0], ph.periodic[1], ph.periodic[2],
                                       make_double3(span[0][0], span[0][1], span[0][2]),
                                       make_double3(span[1][0], span[1][1], span[1][2]),
                                       make_double3(span[2][0], span[2][1], span[2][2]), met[0], met[1], met[2]);
  // Iflag_Gridtype = GRID_AND_JACOBIAN3D: the interior metrics and Jacobian came
  // with the grid (OCFD_mesh.f90:24-26 skips comput_Jacobian3d)
  if (!jac_given) k_jacobian<<<148 * 8, 256, 0, st>>>(g, ph, dc, mp);
  PtrList<double> m10;
  m10.n = 10;
  for (int m = 0; m < 10; m++) m10.p[m] = met[3 + m];
  e = launch_halo(g, ph.periodic, m10, st);
  if (e != cudaSuccess) return e;
  k_jac_ghost_coords<<<148 * 2, 256, 0, st>>>(g, ph, 1, mp);
  k_jac_ghost_coords<<<148 * 2, 256, 0, st>>>(g, ph, 2, mp);
  for (int f = 0; f < 6; f++)
    if (ph.ghost[f] == 2) k_jac_ghost_metrics<<<148 * 2, 256, 0, st>>>(g, ph, f + 1, mp);
  if ((ph.ibc == 3 && ph.ghost[4] == -1) || (ph.ibc == 2 && ph.ghost[2] == -1))
    k_jac_ghost_user<<<148 * 2, 256, 0, st>>>(g, ph, mp);
  k_metric_div<<<148 * 8, 256, 0, st>>>(g.nh, mp);
  return cudaGetLastError();
}

// Which metric arrays are +0.0 (all bits zero) at every point a kernel reads:
// the interior and the face halos (edge and corner halos are never read).  On
// box and 1-D grids the off-diagonal metrics are exact zeros; the face and
// viscous kernels then skip their loads and use the constant (same bits).
// Bit m of *nonzero is set when array m has a nonzero bit pattern there.
__global__ void k_metric_nonzero(Grid G, MetPtrs mp, unsigned int* nonzero) {
  unsigned int mask = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.nh;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % G.nxh) - (LAP - 1), j = (int)((t / G.nxh) % G.nyh) - (LAP - 1);
    const int k = (int)(t / ((long long)G.nxh * G.nyh)) - (LAP - 1);
    const int out = (i < 1 || i > G.nx) + (j < 1 || j > G.ny) + (k < 1 || k > G.nz);
    if (out > 1) continue;
    for (int m = 3; m < 22; m++)
      if (__double_as_longlong(mp.m[m][t]) != 0) mask |= 1u << m;
  }
  mask = __reduce_or_sync(0xffffffffu, mask);
  if ((threadIdx.x & 31) == 0 && mask) atomicOr(nonzero, mask);
}

cudaError_t launch_metric_nonzero(const Grid& g, double* const met[22], unsigned int* nonzero, cudaStream_t st) {
  MetPtrs mp;
  for (int m = 0; m < 22; m++) mp.m[m] = met[m];
  cudaError_t e = cudaMemsetAsync(nonzero, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  k_metric_nonzero<<<148 * 8, 256, 0, st>>>(g, mp, nonzero);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// filtering (OCFD_filtering.f90:4-363), one filter column
__global__ void k_filt_copy(Grid G, int dir, int periodic, const double* src, double* f0) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const double x = src[t];
    f0[G.ih(i, j, k)] = x;
    if (periodic) {  // exchange_boundary_x/y/z of f0 (face halo of this direction only)
      const int l[3] = {i, j, k};
      const int nn = G.len(dir);
      const long long s = G.hstride(dir);
      if (l[dir] <= LAP) f0[G.ih(i, j, k) + nn * s] = x;
      if (l[dir] > nn - LAP) f0[G.ih(i, j, k) - nn * s] = x;
    }
  }
}
__global__ void k_filt_p(Grid G, int dir, int periodic, double gamma, const double* f, double* p) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const double f1 = f[t], f2 = f[t + G.n], f3 = f[t + 2 * G.n], f4 = f[t + 3 * G.n], f5 = f[t + 4 * G.n];
    const double x = (f5 - 0.5 * (f2 * f2 + f3 * f3 + f4 * f4) / f1) * (gamma - 1.0);
    p[G.ih(i, j, k)] = x;
    if (periodic) {
      const int l[3] = {i, j, k};
      const int nn = G.len(dir);
      const long long s = G.hstride(dir);
      if (l[dir] <= LAP) p[G.ih(i, j, k) + nn * s] = x;
      if (l[dir] > nn - LAP) p[G.ih(i, j, k) - nn * s] = x;
    }
  }
}
struct FiltBox {
  int lo[3], hi[3];
};
__device__ __forceinline__ double sc0_at(const double* p, long long s, double rth) {
  const double dp0 = 0.25 * (-p[s] + 2.0 * p[0] - p[-s]);
  const double dp1 = 0.25 * (-p[2 * s] + 2.0 * p[s] - p[0]);
  const double dp2 = 0.25 * (-p[0] + 2.0 * p[-s] - p[-2 * s]);
  const double ri = 0.5 * ((dp0 - dp1) * (dp0 - dp1) + (dp0 - dp2) * (dp0 - dp2)) / (p[0] * p[0]) + 1.0e-16;
  return 0.5 * (1.0 - rth / ri + fabs(1.0 - rth / ri));
}
__global__ void k_filt_apply(Grid G, int dir, int scheme, double s0, double rth, FiltBox B, const double* f0,
                             const double* p, double* fm) {
  const long long ni = B.hi[0] - B.lo[0] + 1, nj = B.hi[1] - B.lo[1] + 1, nk = B.hi[2] - B.lo[2] + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  const long long s = G.hstride(dir);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ni * nj * nk; t += (long long)gridDim.x * blockDim.x) {
    const int i = B.lo[0] + (int)(t % ni), j = B.lo[1] + (int)((t / ni) % nj), k = B.lo[2] + (int)(t / (ni * nj));
    const long long c = G.ih(i, j, k);
    const double* q = f0 + c;
    double r;
    if (scheme == 1) {
      const double d0 = 0.243527493120, d1 = -0.204788880640, d2 = 0.120007591680, d3 = -0.045211119360,
                   d4 = 0.008228661760;
      r = q[0] - s0 * (d0 * q[0] + d1 * (q[-s] + q[s]) + d2 * (q[-2 * s] + q[2 * s]) + d3 * (q[-3 * s] + q[3 * s]) +
                       d4 * (q[-4 * s] + q[4 * s]));
    } else {
      const double c1 = -0.210383, c2 = 0.039617;
      const double sa = sc0_at(p + c, s, rth), sp = sc0_at(p + c + s, s, rth), sm = sc0_at(p + c - s, s, rth);
      const double sc1 = 0.5 * (sa + sp), sc2 = 0.5 * (sa + sm);
      r = q[0] - s0 * (sc1 * (c1 * (q[s] - q[0]) + c2 * (q[2 * s] - q[-s])) -
                       sc2 * (c1 * (q[0] - q[-s]) + c2 * (q[s] - q[-2 * s])));
    }
    fm[G.ii(i, j, k)] = r;
  }
}

cudaError_t launch_filter(const Grid& g, const Phys& ph, double* f, double* scratch, const double* F,
                          cudaStream_t st) {
  double* f0 = scratch;
  double* p = scratch + g.nh;
  const int nn[3] = {g.nx, g.ny, g.nz};
  int lo[3] = {(int)llround(F[4]), (int)llround(F[6]), (int)llround(F[8])};
  int hi[3] = {(int)llround(F[5]), (int)llround(F[7]), (int)llround(F[9])};
  for (int d = 0; d < 3; d++) {
    if (lo[d] < 1) lo[d] = 1;
    if (hi[d] > nn[d]) hi[d] = nn[d];
  }
  const int scheme = (int)llround(F[10]);
  const double s0 = F[11], rth = F[12];
  for (int d = 0; d < 3; d++) {
    if ((int)llround(F[1 + d]) != 1) continue;
    if (scheme != 1 && scheme != 2) continue;
    FiltBox B;
    for (int q = 0; q < 3; q++) {
      B.lo[q] = lo[q];
      B.hi[q] = hi[q];
    }
    if (!ph.periodic[d]) {  // OCFD_filtering.f90:84-85 / :198-199
      const int m = scheme == 1 ? 6 : 4;
      if (B.lo[d] < m) B.lo[d] = m;
      if (B.hi[d] > nn[d] - (m - 1)) B.hi[d] = nn[d] - (m - 1);
    }
    if (scheme == 2) k_filt_p<<<148 * 8, 256, 0, st>>>(g, d, ph.periodic[d], ph.gamma, f, p);
    for (int m = 0; m < 5; m++) {
      k_filt_copy<<<148 * 8, 256, 0, st>>>(g, d, ph.periodic[d], f + m * g.n, f0);
      k_filt_apply<<<148 * 8, 256, 0, st>>>(g, d, scheme, s0, rth, B, f0, p, f + m * g.n);
    }
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// show_flow_msg sums (OCFD_Time_Adv.f90:75-86)
__global__ void __launch_bounds__(RED_THREADS) k_flow_msg(Grid G, Phys ph, const double* f, const double* d,
                                                          const double* u, const double* v, const double* w,
                                                          const double* T, const double* ajac, double* part) {
  __shared__ double sm[3 * RED_THREADS];
  const double p00 = 1.0 / (ph.gamma * ph.ma * ph.ma);
  const double tmp1 = 1.0 - ph.gamma;
  double s[3] = {0.0, 0.0, 0.0};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    const double tmp0 = 1.0 / ajac[c];
    const double dd = d[c], uu = u[c], vv = v[c], ww = w[c];
    s[0] += f[t + 4 * G.n] * tmp0;
    s[1] += dd * (uu * uu + vv * vv + ww * ww) * 0.5 * tmp0;
    s[2] += p00 * pow(dd, tmp1) * T[c] * tmp0;
  }
  block_sum<3>(s, sm);
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) part[blockIdx.x * 3 + q] = s[q];
}

cudaError_t launch_flow_msg(const Grid& g, const Phys& ph, const double* f, double* const prim[5],
                            const double* ajac, double* scratch, double* out3, cudaStream_t st) {
  k_flow_msg<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, ph, f, prim[0], prim[1], prim[2], prim[3], prim[4], ajac, scratch);
  k_final_sum<3><<<1, RED_THREADS, 0, st>>>(scratch, RED_BLOCKS, out3);
  return cudaGetLastError();
}

// ana_box sums (OCFD_ANA.f90:209-247) and the d_rms pass (:277-287)
__global__ void __launch_bounds__(RED_THREADS) k_ana_box(Grid G, Phys ph, DCoef dc, const double* d, const double* u,
                                                         const double* v, const double* w, const double* T,
                                                         MetPtrs mp, double* part) {
  __shared__ double sm[14 * RED_THREADS];
  double s[14];
  for (int q = 0; q < 14; q++) s[q] = 0.0;
  const int cd8 = ph.scheme_vis == 6;
  double* const* M = mp.m;
  const double Tsb = 110.4 / ph.ref_amu_t0, TmpR = 1.0 / ph.re;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    const long long st[3] = {1, (long long)G.nxh, (long long)G.nxh * G.nyh};
    const int l[3] = {i, j, k};
    const double* q3[3] = {u, v, w};
    double gr[3][3];
    for (int q = 0; q < 3; q++)
      for (int dd = 0; dd < 3; dd++) gr[q][dd] = d0h(q3[q] + c, st[dd], l[dd], G.len(dd), ph.periodic[dd], cd8, dc, dd);
    const double Akx = M[3][c], Aky = M[4][c], Akz = M[5][c], Aix = M[6][c], Aiy = M[7][c], Aiz = M[8][c];
    const double Asx = M[9][c], Asy = M[10][c], Asz = M[11][c];
    const double ux = gr[0][0] * Akx + gr[0][1] * Aix + gr[0][2] * Asx;
    const double uy = gr[0][0] * Aky + gr[0][1] * Aiy + gr[0][2] * Asy;
    const double uz = gr[0][0] * Akz + gr[0][1] * Aiz + gr[0][2] * Asz;
    const double vx = gr[1][0] * Akx + gr[1][1] * Aix + gr[1][2] * Asx;
    const double vz = gr[1][0] * Akz + gr[1][1] * Aiz + gr[1][2] * Asz;
    const double vy = gr[1][0] * Aky + gr[1][1] * Aiy + gr[1][2] * Asy;
    const double wx = gr[2][0] * Akx + gr[2][1] * Aix + gr[2][2] * Asx;
    const double wy = gr[2][0] * Aky + gr[2][1] * Aiy + gr[2][2] * Asy;
    (void)vy;
    const double TT = T[c], dd = d[c], uu = u[c], vv = v[c], ww = w[c];
    const double amu = TmpR * (1.0 + Tsb) * sqrt(TT * TT * TT) / (Tsb + TT);
    s[0] += uu * uu;
    s[1] += vv * vv;
    s[2] += ww * ww;
    s[3] += ux * ux;
    s[4] += ux * ux * ux;
    s[5] += (ux * ux) * (ux * ux);
    s[6] += dd;
    s[7] += sqrt(TT) / ph.ma;
    s[8] += amu;
    s[9] += (uu * uu + vv * vv + ww * ww) * dd * 0.5;
    s[10] += TT;
    s[11] += uu * uu * uu;
    s[12] += (uu * uu) * (uu * uu);
    s[13] += (wy - vz) * (wy - vz) + (uz - wx) * (uz - wx) + (vx - uy) * (vx - uy);
  }
  block_sum<14>(s, sm);
  if (threadIdx.x == 0)
    for (int q = 0; q < 14; q++) part[blockIdx.x * 14 + q] = s[q];
}
__global__ void __launch_bounds__(RED_THREADS) k_drms(Grid G, const double* d, const double* sums, double* part) {
  __shared__ double sm[RED_THREADS];
  const double d_aver = sums[6] / (double)(G.nx * G.ny * G.nz);
  double s[1] = {0.0};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const double x = d[G.ih(i, j, k)] - d_aver;
    s[0] += x * x;
  }
  block_sum<1>(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

cudaError_t launch_ana_box(const Grid& g, const Phys& ph, const DCoef& dc, double* const prim[5],
                           const double* const met[22], double* scratch, double* out14, double* out_drms,
                           cudaStream_t st) {
  MetPtrs mp;
  for (int m = 0; m < 22; m++) mp.m[m] = const_cast<double*>(met[m]);
  k_ana_box<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, ph, dc, prim[0], prim[1], prim[2], prim[3], prim[4], mp, scratch);
  k_final_sum<14><<<1, RED_THREADS, 0, st>>>(scratch, RED_BLOCKS, out14);
  k_drms<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, prim[0], out14, scratch);
  k_final_sum<1><<<1, RED_THREADS, 0, st>>>(scratch, RED_BLOCKS, out_drms);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Analysis of OCFD_analysis (OCFD_ANA.f90:3-31) beyond ana_box.

// ana_getQ (OCFD_ANA.f90:127-171): Q = II(grad u) from the CD6/CD8 derivatives of
// u, v, w (halos exchanged by the caller) and the metrics.
__global__ void k_ana_q(Grid G, Phys ph, DCoef dc, const double* u, const double* v, const double* w, MetPtrs mp,
                        double* q) {
  const int cd8 = ph.scheme_vis == 6;
  double* const* M = mp.m;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    const long long st[3] = {1, (long long)G.nxh, (long long)G.nxh * G.nyh};
    const int l[3] = {i, j, k};
    const double* q3[3] = {u, v, w};
    double gr[3][3];
    for (int a = 0; a < 3; a++)
      for (int dd = 0; dd < 3; dd++) gr[a][dd] = d0h(q3[a] + c, st[dd], l[dd], G.len(dd), ph.periodic[dd], cd8, dc, dd);
    const double Akx = M[3][c], Aky = M[4][c], Akz = M[5][c], Aix = M[6][c], Aiy = M[7][c], Aiz = M[8][c];
    const double Asx = M[9][c], Asy = M[10][c], Asz = M[11][c];
    const double ux = gr[0][0] * Akx + gr[0][1] * Aix + gr[0][2] * Asx;
    const double vx = gr[1][0] * Akx + gr[1][1] * Aix + gr[1][2] * Asx;
    const double wx = gr[2][0] * Akx + gr[2][1] * Aix + gr[2][2] * Asx;
    const double uy = gr[0][0] * Aky + gr[0][1] * Aiy + gr[0][2] * Asy;
    const double vy = gr[1][0] * Aky + gr[1][1] * Aiy + gr[1][2] * Asy;
    const double wy = gr[2][0] * Aky + gr[2][1] * Aiy + gr[2][2] * Asy;
    const double uz = gr[0][0] * Akz + gr[0][1] * Aiz + gr[0][2] * Asz;
    const double vz = gr[1][0] * Akz + gr[1][1] * Aiz + gr[1][2] * Asz;
    const double wz = gr[2][0] * Akz + gr[2][1] * Aiz + gr[2][2] * Asz;
    q[t] = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
  }
}
cudaError_t launch_ana_q(const Grid& g, const Phys& ph, const DCoef& dc, double* const prim[5],
                         const double* const met[22], double* q, cudaStream_t st) {
  MetPtrs mp;
  for (int m = 0; m < 22; m++) mp.m[m] = const_cast<double*>(met[m]);
  k_ana_q<<<148 * 8, 256, 0, st>>>(g, ph, dc, prim[1], prim[2], prim[3], mp, q);
  return cudaGetLastError();
}

// ana_time_average (OCFD_ANA.f90:34-125): running mean of d, u, v, w, T over the
// K samples taken so far, mean = (K mean + q) / (K + 1).
__global__ void k_ana_average(Grid G, const double* d, const double* u, const double* v, const double* w,
                              const double* T, double* mean, double K) {
  const double* Q[5] = {d, u, v, w, T};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode(G, t, i, j, k);
    const long long c = G.ih(i, j, k);
    for (int a = 0; a < 5; a++) mean[t + a * G.n] = (K * mean[t + a * G.n] + Q[a][c]) / (K + 1.0);
  }
}
cudaError_t launch_ana_average(const Grid& g, double* const prim[5], double* mean, int K, cudaStream_t st) {
  k_ana_average<<<148 * 8, 256, 0, st>>>(g, prim[0], prim[1], prim[2], prim[3], prim[4], mean, (double)K);
  return cudaGetLastError();
}

// Ana_corner (OCFD_ANA.f90:316-384): per i, span averages of the wall-tangential
// velocity and temperature at j = 2 and of the wall pressure, in the reference's
// k order (one thread per i).
__global__ void k_ana_corner(Grid G, Phys ph, const double* d, const double* u, const double* v, const double* T,
                             const double* axx, const double* ayy, double* out) {
  const double p00 = 1.0 / (ph.gamma * ph.ma * ph.ma);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i <= G.nx; i += gridDim.x * blockDim.x) {
    double sx, sy;
    if (i < G.nx) {
      sx = axx[G.ih(i + 1, 1, 1)] - axx[G.ih(i, 1, 1)];
      sy = ayy[G.ih(i + 1, 1, 1)] - ayy[G.ih(i, 1, 1)];
    } else {
      sx = axx[G.ih(G.nx, 1, 1)] - axx[G.ih(G.nx - 1, 1, 1)];
      sy = ayy[G.ih(G.nx, 1, 1)] - ayy[G.ih(G.nx - 1, 1, 1)];
    }
    const double tmp = 1.0 / sqrt(sx * sx + sy * sy);
    sx = sx * tmp;
    sy = sy * tmp;
    double us = 0.0, Ts = 0.0, ps = 0.0;
    for (int k = 1; k <= G.nz; k++) {
      const long long c2 = G.ih(i, 2, k), c1 = G.ih(i, 1, k);
      us = us + u[c2] * sx + v[c2] * sy;
      Ts = Ts + T[c2];
      ps = ps + p00 * d[c1] * T[c1];
    }
    const double r = 1.0 / G.nz;
    out[i - 1] = us * r;
    out[G.nx + i - 1] = Ts * r;
    out[2 * G.nx + i - 1] = ps * r;
  }
}
cudaError_t launch_ana_corner(const Grid& g, const Phys& ph, double* const prim[5], const double* axx,
                              const double* ayy, double* out, cudaStream_t st) {
  k_ana_corner<<<(g.nx + 255) / 256, 256, 0, st>>>(g, ph, prim[0], prim[1], prim[2], prim[4], axx, ayy, out);
  return cudaGetLastError();
}

// A box [ib,ie] x [jb,je] x [kb,ke] (1-based, inclusive) of a haloed array, i fastest.
__global__ void k_gather_box(Grid G, const double* src, int ib, int jb, int kb, int ni, int nj, int nk, double* dst) {
  const long long tot = (long long)ni * nj * nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % ni), b = (int)((t / ni) % nj), c = (int)(t / ((long long)ni * nj));
    dst[t] = src[G.ih(ib + a, jb + b, kb + c)];
  }
}
cudaError_t launch_gather_box(const Grid& g, const double* src, int ib, int ie, int jb, int je, int kb, int ke,
                              double* dst, cudaStream_t st) {
  k_gather_box<<<148 * 4, 256, 0, st>>>(g, src, ib, jb, kb, ie - ib + 1, je - jb + 1, ke - kb + 1, dst);
  return cudaGetLastError();
}

}  // namespace ocfd
