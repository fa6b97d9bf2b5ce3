// Synthetic helical scans: FP64 line integrals through an ellipsoid phantom,
// Poisson noise and log transform. This is the project's test-data generator;
// the reference reads measured DICOM-CT-PD frames instead
// (modules/fct_read/src/DicomDataSet.cpp:56-155).
#include "wfbp_internal.h"

namespace {

constexpr int MAX_ELLIPSOIDS = 128;
__constant__ wfbp_ellipsoid c_ell[MAX_ELLIPSOIDS];

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of the two 32x32->64 multiplies with
// key schedule increments 0x9E3779B9 / 0xBB67AE85.
__device__ void philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                           uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__device__ __forceinline__ double u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

// Inversion by sequential search below mean 64, rounded normal approximation above.
__device__ double poisson_draw(double lam, const uint32_t r[4]) {
  if (lam <= 0) return 0.0;
  if (lam < 64.0) {
    double u = u01(r[0]), pk = exp(-lam), F = pk;
    int k = 0;
    while (u > F && k < 4096) { k++; pk *= lam / k; F += pk; }
    return (double)k;
  }
  double z = sqrt(-2.0 * log(u01(r[0]))) * cos(2.0 * 3.141592653589793 * u01(r[1]));
  double n = floor(lam + sqrt(lam) * z + 0.5);
  return n < 0 ? 0.0 : n;
}

// Ray of reading v, raw row r, raw channel k in the conventions the
// reference's rebin and backprojection invert (cuda_kernels.cuh:11-39,
// 198-287): tube angle and table position decrease with the reading index,
// flipped channel b = nch-1-k has fan angle beta = (b - c0) dcol / sdd, the
// parallel direction is theta = angle - beta, the in-plane ray is
// x sin(theta) - y cos(theta) = (nch + 1.75 - 2 c0) ds - R sin(beta) (the
// p-flip of cuda_kernels.cuh:251), its source sits on the circle of radius R,
// and flipped row rr = nr-1-r rises by (rr - (nr-1)/2) drow / sdd per mm.
__global__ void k_synth(wfbp_synth_scan s, int ne, float* __restrict__ out) {
  const long total = (long)s.n_readings * s.rows * s.channels;
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= total) return;
  const int k = (int)(id % s.channels);
  const long row = id / s.channels;
  const int r = (int)(row % s.rows);
  const long v = row / s.rows;
  const int nch = s.channels, nr = s.rows;
  // flying focal spot: reading v of focal state (sp, sz) samples effective
  // channel 2b + sp and effective row 2rr + sz of a detector with twice the
  // channels / rows at half the spacing and central channel 2 c0 + 1/2
  const int phi = (s.ffs_mode & WFBP_FFS_PHI) != 0, zf = (s.ffs_mode & WFBP_FFS_Z) != 0;
  const int G = (phi ? 2 : 1) * (zf ? 2 : 1);
  const int rho = (int)(v % G);
  const int spf = phi ? (G == 4 ? (rho & 1) : rho) : 0, szf = zf ? (G == 4 ? (rho >> 1) : rho) : 0;
  const int nche = phi ? 2 * nch : nch, nre = zf ? 2 * nr : nr;
  const double c0e = phi ? 2.0 * s.central_channel + 0.5 : s.central_channel;
  const double dcole = phi ? 0.5 * s.dcol : s.dcol, drowe = zf ? 0.5 * s.drow : s.drow;
  const double R = s.sid;
  const double ds = dcole * R / s.sdd;
  const double delta = nche + 1.75 - 2.0 * c0e;
  const int b = nch - 1 - k, rr = nr - 1 - r;
  const int be = phi ? 2 * b + spf : b, rre = zf ? 2 * rr + szf : rr;
  const double beta = (be - c0e) * dcole / s.sdd;
  const double ang = s.angle0 + v * s.dangle;
  const double zs = s.z0 + v * s.dz;
  const double theta = ang - beta;
  double sn, cs;
  sincos(theta, &sn, &cs);
  const double pstar = delta * ds - R * sin(beta);
  const double tt = sqrt(R * R - pstar * pstar);
  const double S0 = pstar * sn + tt * cs, S1 = -pstar * cs + tt * sn, S2 = zs;
  const double U0 = -cs, U1 = -sn, U2 = (rre - (nre - 1) / 2.0) * drowe / s.sdd;
  const double unorm = sqrt(U0 * U0 + U1 * U1 + U2 * U2);
  double p = 0.0;
  for (int n = 0; n < ne; n++) {
    const wfbp_ellipsoid e = c_ell[n];
    double sp, cp;
    sincos(e.phi, &sp, &cp);
    const double dx = S0 - e.cx, dy = S1 - e.cy, dzz = S2 - e.cz;
    const double px = (dx * cp + dy * sp) / e.ax, py = (-dx * sp + dy * cp) / e.ay, pz = dzz / e.az;
    const double ux = (U0 * cp + U1 * sp) / e.ax, uy = (-U0 * sp + U1 * cp) / e.ay, uz = U2 / e.az;
    const double A = ux * ux + uy * uy + uz * uz, B = px * ux + py * uy + pz * uz,
                 C = px * px + py * py + pz * pz - 1.0;
    const double disc = B * B - A * C;
    if (disc > 0) p += e.mu * (2.0 * sqrt(disc) / A) * unorm;
  }
  if (s.i0 > 0) {
    const uint64_t idx = (uint64_t)row * nch + k;
    uint32_t rnd[4];
    philox4x32((uint32_t)idx, (uint32_t)(idx >> 32), 0u, 0u, (uint32_t)s.seed, (uint32_t)(s.seed >> 32), rnd);
    double n = poisson_draw(s.i0 * exp(-p), rnd);
    if (n < 1.0) n = 1.0;
    p = -log(n / s.i0);
  }
  out[id] = (float)p;
}

}  // namespace

cudaError_t launch_synth(const wfbp_synth_scan& scan, const wfbp_ellipsoid* h_e, int ne, float* out,
                         cudaStream_t s) {
  if (ne > MAX_ELLIPSOIDS) return cudaErrorInvalidValue;
  cudaError_t e = cudaSuccess;
  if (ne > 0) e = cudaMemcpyToSymbolAsync(c_ell, h_e, sizeof(wfbp_ellipsoid) * ne, 0, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  long total = (long)scan.n_readings * scan.rows * scan.channels;
  k_synth<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(scan, ne, out);
  return cudaGetLastError();
}
