/*
 * orc_impl.h -- body of the CPU oracle, included twice by broccoli_oracle.c
 * with REAL = float / SFX = _f32 and REAL = double / SFX = _f64.
 *
 * TEST INFRASTRUCTURE ONLY (see broccoli_oracle.h).  Each function restates
 * one piece of the reference and cites the file:line it follows; paths are
 * relative to the BROCCOLI source tree.  The float build keeps the
 * reference's operation order (per-slice partial sums, per-row / per-column /
 * per-slice reduction order) so that it is the FP32 parity target; the double
 * build is the same algorithm in double precision.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

#if REAL_IS_FLOAT
#define RSQRT(x) sqrtf(x)
#define RATAN2(y, x) atan2f(y, x)
#define RCOS(x) cosf(x)
#define RFLOOR(x) floorf(x)
#define RHALF 0.5f
#define RONE 1.0f
#define RZERO 0.0f
#else
#define RSQRT(x) sqrt(x)
#define RATAN2(y, x) atan2(y, x)
#define RCOS(x) cos(x)
#define RFLOOR(x) floor(x)
#define RHALF 0.5
#define RONE 1.0
#define RZERO 0.0
#endif

/* Non-separable 3D filtering with nfilt complex 7x7x7 filters.
 * Follows BROCCOLI_LIB::NonseparableConvolution3D (code/BROCCOLI_LIB/
 * broccoli_lib.cpp:4974-5027): responses are zeroed, then for z-offsets
 * -3..+3 (filter slice zz = 6..0) a 2D 7x7 pass over the slice z+zoff is
 * accumulated.  The 2D pass is kernelConvolution.cpp:2802-2867: the filter
 * index runs 6..0 while the offset runs -3..+3 (a true convolution), with
 * zero padding outside the volume.  `filters` holds nfilt x {re[343],
 * im[343]}; `out` holds nfilt interleaved complex volumes. */
void FN(orc_filter3d)(const REAL* vol, int W, int H, int D, const REAL* filters,
                      int nfilt, REAL* out) {
  const long V = (long)W * H * D;
  for (int f = 0; f < nfilt; f++)
    for (long i = 0; i < 2 * V; i++) out[(long)f * 2 * V + i] = RZERO;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++) {
    REAL s[2 * 6];
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const long idx = x + (long)y * W + (long)z * W * H;
        for (int zz = 6; zz >= 0; zz--) {
          const int zoff = 3 - zz;
          const int zi = z + zoff;
          for (int k = 0; k < 2 * nfilt; k++) s[k] = RZERO;
          if (zi >= 0 && zi < D) {
            for (int fy = 6; fy >= 0; fy--) {
              const int yi = y + 3 - fy;
              if (yi < 0 || yi >= H) continue;
              for (int fx = 6; fx >= 0; fx--) {
                const int xi = x + 3 - fx;
                if (xi < 0 || xi >= W) continue;
                const REAL pixel = vol[xi + (long)yi * W + (long)zi * W * H];
                const int tap = fx + fy * 7 + zz * 49;
                for (int f = 0; f < nfilt; f++) {
                  s[2 * f] += filters[f * 686 + tap] * pixel;
                  s[2 * f + 1] += filters[f * 686 + 343 + tap] * pixel;
                }
              }
            }
          }
          for (int f = 0; f < nfilt; f++) {
            out[(long)f * 2 * V + 2 * idx] += s[2 * f];
            out[(long)f * 2 * V + 2 * idx + 1] += s[2 * f + 1];
          }
        }
      }
  }
}

/* Phase difference arg(q1 conj q2) and certainty |q1 q2| cos^2(dphi/2).
 * kernelRegistration.cpp:173-211. */
void FN(orc_phase_diff_cert)(const REAL* q1, const REAL* q2, long V, REAL* pd,
                             REAL* cert) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < V; i++) {
    const REAL ax = q1[2 * i], ay = q1[2 * i + 1];
    const REAL cx = q2[2 * i], cy = q2[2 * i + 1];
    REAL re = ax * cx + ay * cy;
    REAL im = ay * cx - ax * cy;
    const REAL d = RATAN2(im, re);
    re = ax * cx - ay * cy;
    im = ay * cx + ax * cy;
    const REAL c = RCOS(d * RHALF);
    pd[i] = d;
    cert[i] = RSQRT(re * re + im * im) * c * c;
  }
}

/* Phase gradient along `axis` (0=x,1=y,2=z): arg of the sum of the four
 * neighbour products q[+1] conj q[0] + q[0] conj q[-1] of both responses.
 * kernelRegistration.cpp:213-382.  The first and last sample along the axis
 * are left unwritten, as in the reference. */
void FN(orc_phase_grad)(const REAL* q1, const REAL* q2, int axis, int W, int H,
                        int D, REAL* grad) {
  const long step = axis == 0 ? 1 : (axis == 1 ? (long)W : (long)W * H);
  const int n = axis == 0 ? W : (axis == 1 ? H : D);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const int c = axis == 0 ? x : (axis == 1 ? y : z);
        if (c - 1 < 0 || c + 1 >= n) continue;
        const long i = x + (long)y * W + (long)z * W * H;
        const long ip = i + step, im = i - step;
        REAL tr = RZERO, ti = RZERO;
        const REAL* qs[2] = {q1, q2};
        for (int k = 0; k < 2; k++) {
          const REAL* q = qs[k];
          REAL ax = q[2 * ip], ay = q[2 * ip + 1];
          REAL cx = q[2 * i], cy = q[2 * i + 1];
          tr += ax * cx + ay * cy;
          ti += ay * cx - ax * cy;
          ax = cx;
          ay = cy;
          cx = q[2 * im];
          cy = q[2 * im + 1];
          tr += ax * cx + ay * cy;
          ti += ay * cx - ax * cy;
        }
        grad[i] = RATAN2(ti, tr);
      }
}

/* (row, column) of the 10 A-matrix entries filled by one axis, in the order
 * of the monomials [1, x, y, z, xx, xy, xz, yy, yz, zz].  This is the table
 * of GetParameterIndices (kernelRegistration.cpp:43-171): axis k owns the
 * parameters {k, 3+3k, 4+3k, 5+3k}. */
static void FN(orc_axis_entry)(int axis, int e, int* i, int* j) {
  static const int mono_a[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
  static const int mono_b[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
  const int param[4] = {axis, 3 + 3 * axis, 4 + 3 * axis, 5 + 3 * axis};
  *i = param[mono_a[e]];
  *j = param[mono_b[e]];
}

/* Sums of c g^2 [1,x,y,z,xx,xy,xz,yy,yz,zz] and c g dphi [1,x,y,z] over the
 * interior (border (filter_size-1)/2 in every axis), coordinates relative to
 * the volume centre.  Order of summation as in the reference: along x per
 * (y,z) row (kernelRegistration.cpp:387-485), then over y per z
 * (:695-720, :750-776), then over z (:723-747, :780-800).  Writes the 10
 * lower-triangle entries of A (column-major 12x12, A[i + 12 j]) and the 4
 * entries of h that belong to this axis. */
void FN(orc_ah_axis)(const REAL* pd, const REAL* grad, const REAL* cert,
                     int axis, int W, int H, int D, int filter_size, REAL* A144,
                     REAL* h12) {
  const int b = (filter_size - 1) / 2;
  REAL A[10], h[4];
  for (int e = 0; e < 10; e++) A[e] = RZERO;
  for (int e = 0; e < 4; e++) h[e] = RZERO;
  for (int z = b; z < D - b; z++) {
    REAL A1[10], h1[4];
    for (int e = 0; e < 10; e++) A1[e] = RZERO;
    for (int e = 0; e < 4; e++) h1[e] = RZERO;
    for (int y = b; y < H - b; y++) {
      const REAL yf = (REAL)y - ((REAL)H - RONE) * RHALF;
      const REAL zf = (REAL)z - ((REAL)D - RONE) * RHALF;
      REAL a[10], hv[4];
      for (int e = 0; e < 10; e++) a[e] = RZERO;
      for (int e = 0; e < 4; e++) hv[e] = RZERO;
      for (int x = b; x < W - b; x++) {
        const REAL xf = (REAL)x - ((REAL)W - RONE) * RHALF;
        const long i = x + (long)y * W + (long)z * W * H;
        const REAL d = pd[i], g = grad[i], c = cert[i];
        const REAL cgg = c * g * g;
        const REAL cgd = c * g * d;
        a[0] += cgg;
        a[1] += xf * cgg;
        a[2] += yf * cgg;
        a[3] += zf * cgg;
        a[4] += xf * xf * cgg;
        a[5] += xf * yf * cgg;
        a[6] += xf * zf * cgg;
        a[7] += yf * yf * cgg;
        a[8] += yf * zf * cgg;
        a[9] += zf * zf * cgg;
        hv[0] += cgd;
        hv[1] += xf * cgd;
        hv[2] += yf * cgd;
        hv[3] += zf * cgd;
      }
      for (int e = 0; e < 10; e++) A1[e] += a[e];
      for (int e = 0; e < 4; e++) h1[e] += hv[e];
    }
    for (int e = 0; e < 10; e++) A[e] += A1[e];
    for (int e = 0; e < 4; e++) h[e] += h1[e];
  }
  for (int e = 0; e < 10; e++) {
    int i, j;
    FN(orc_axis_entry)(axis, e, &i, &j);
    A144[i + 12 * j] = A[e];
  }
  h12[axis] = h[0];
  h12[3 + 3 * axis] = h[1];
  h12[4 + 3 * axis] = h[2];
  h12[5 + 3 * axis] = h[3];
}

/* The 12x12 normal equations of one affine iteration from the three pairs of
 * responses (q1: reference, q2: aligned volume; each 3 interleaved complex
 * volumes).  Follows the kernel sequence of AlignTwoVolumesLinear
 * (broccoli_lib.cpp:5315-5381) and the mirroring of :5384-5392.  A is
 * returned full and symmetric, column-major. */
void FN(orc_normal_equations)(const REAL* q1, const REAL* q2, int W, int H,
                              int D, REAL* A144, REAL* h12) {
  const long V = (long)W * H * D;
  REAL* pd = (REAL*)calloc(V, sizeof(REAL));
  REAL* cert = (REAL*)calloc(V, sizeof(REAL));
  REAL* grad = (REAL*)calloc(V, sizeof(REAL));
  for (int e = 0; e < 144; e++) A144[e] = RZERO;
  for (int e = 0; e < 12; e++) h12[e] = RZERO;
  for (int axis = 0; axis < 3; axis++) {
    const REAL* a = q1 + (long)axis * 2 * V;
    const REAL* c = q2 + (long)axis * 2 * V;
    FN(orc_phase_diff_cert)(a, c, V, pd, cert);
    FN(orc_phase_grad)(a, c, axis, W, H, D, grad);
    FN(orc_ah_axis)(pd, grad, cert, axis, W, H, D, 7, A144, h12);
  }
  for (int j = 0; j < 12; j++)
    for (int i = 0; i < 12; i++) A144[j + i * 12] = A144[i + j * 12];
  free(pd);
  free(cert);
  free(grad);
}

/* Normal equations with the certainties smoothed first by a separable
 * 3x3x3 Gaussian (sigma in voxels, weights exp(-1/2sigma^2), 1, exp(...)
 * normalised).  Not in the reference (its linear path uses the raw
 * certainties); this is the certainty-smoothing switch of the batched
 * motion-correction workload, specified here.  Interior voxels only, so
 * every neighbour is inside the volume. */
void FN(orc_normal_equations_smoothcert)(const REAL* q1, const REAL* q2, int W, int H, int D,
                                         double sigma, REAL* A144, REAL* h12) {
  const long V = (long)W * H * D;
  REAL* pd = (REAL*)calloc(V, sizeof(REAL));
  REAL* cert = (REAL*)calloc(V, sizeof(REAL));
  REAL* cs = (REAL*)calloc(V, sizeof(REAL));
  REAL* grad = (REAL*)calloc(V, sizeof(REAL));
  const float e = (float)exp(-1.0 / (2.0 * sigma * sigma));
  const REAL w0 = (REAL)(1.0f / (1.0f + 2.0f * e));
  const REAL w1 = (REAL)(e * (1.0f / (1.0f + 2.0f * e)));
  const REAL w[3] = {w1, w0, w1};
  for (int e2 = 0; e2 < 144; e2++) A144[e2] = RZERO;
  for (int e2 = 0; e2 < 12; e2++) h12[e2] = RZERO;
  for (int axis = 0; axis < 3; axis++) {
    const REAL* a = q1 + (long)axis * 2 * V;
    const REAL* c = q2 + (long)axis * 2 * V;
    FN(orc_phase_diff_cert)(a, c, V, pd, cert);
    FN(orc_phase_grad)(a, c, axis, W, H, D, grad);
    for (int z = 1; z < D - 1; z++)
      for (int y = 1; y < H - 1; y++)
        for (int x = 1; x < W - 1; x++) {
          REAL s = RZERO;
          for (int dz = -1; dz <= 1; dz++) {
            REAL sy = RZERO;
            for (int dy = -1; dy <= 1; dy++) {
              const long r = x + (long)(y + dy) * W + (long)(z + dz) * W * H;
              const REAL sx = w1 * cert[r - 1] + w0 * cert[r] + w1 * cert[r + 1];
              sy += w[dy + 1] * sx;
            }
            s += w[dz + 1] * sy;
          }
          cs[x + (long)y * W + (long)z * W * H] = s;
        }
    FN(orc_ah_axis)(pd, grad, cs, axis, W, H, D, 7, A144, h12);
  }
  for (int j = 0; j < 12; j++)
    for (int i = 0; i < 12; i++) A144[j + i * 12] = A144[i + j * 12];
  free(pd);
  free(cert);
  free(cs);
  free(grad);
}

/* p = A^-1 h in double precision, A column-major n x n, result rounded to
 * `real`.  The reference uses Eigen's full-pivoting Householder QR
 * (SolveEquationSystem, broccoli_lib.cpp:17157-17186); this is Gaussian
 * elimination with complete pivoting, which gives the same solution to
 * double rounding.  Rank handling follows the same rule: pivots below
 * eps * n * |largest pivot| are treated as zero and the matching unknowns are
 * set to 0 (a zero matrix gives p = 0). */
void FN(orc_solve)(const REAL* Ain, const REAL* hin, int n, REAL* p) {
  double A[144], h[12], x[12];
  int colperm[12];
  for (int i = 0; i < n; i++) {
    h[i] = (double)hin[i];
    colperm[i] = i;
    for (int j = 0; j < n; j++) A[i * n + j] = (double)Ain[i + j * n];
  }
  double maxpiv = 0.0;
  int rank = 0;
  for (int k = 0; k < n; k++) {
    int pr = k, pc = k;
    double best = -1.0;
    for (int i = k; i < n; i++)
      for (int j = k; j < n; j++)
        if (fabs(A[i * n + j]) > best) {
          best = fabs(A[i * n + j]);
          pr = i;
          pc = j;
        }
    if (k == 0) maxpiv = best;
    if (best <= maxpiv * 2.220446049250313e-16 * n || best == 0.0) break;
    rank++;
    if (pr != k) {
      for (int j = 0; j < n; j++) {
        double t = A[k * n + j];
        A[k * n + j] = A[pr * n + j];
        A[pr * n + j] = t;
      }
      double t = h[k];
      h[k] = h[pr];
      h[pr] = t;
    }
    if (pc != k) {
      for (int i = 0; i < n; i++) {
        double t = A[i * n + k];
        A[i * n + k] = A[i * n + pc];
        A[i * n + pc] = t;
      }
      int t = colperm[k];
      colperm[k] = colperm[pc];
      colperm[pc] = t;
    }
    for (int i = k + 1; i < n; i++) {
      const double m = A[i * n + k] / A[k * n + k];
      if (m == 0.0) continue;
      for (int j = k; j < n; j++) A[i * n + j] -= m * A[k * n + j];
      h[i] -= m * h[k];
    }
  }
  double y[12];
  for (int i = 0; i < n; i++) y[i] = 0.0;
  for (int i = rank - 1; i >= 0; i--) {
    double s = h[i];
    for (int j = i + 1; j < rank; j++) s -= A[i * n + j] * y[j];
    y[i] = s / A[i * n + i];
  }
  for (int i = 0; i < n; i++) x[colperm[i]] = y[i];
  for (int i = 0; i < n; i++) p[i] = (REAL)x[i];
}

/* Polar factor U V^T of a 3x3 matrix from its SVD, by one-sided (Hestenes)
 * Jacobi sweeps in double.  M is row-major. */
static void FN(orc_polar3)(const double* M, double* R) {
  double A[9], Vm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 9; i++) A[i] = M[i];
  for (int sweep = 0; sweep < 60; sweep++) {
    int rotated = 0;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double al = 0, be = 0, ga = 0;
        for (int i = 0; i < 3; i++) {
          al += A[i * 3 + p] * A[i * 3 + p];
          be += A[i * 3 + q] * A[i * 3 + q];
          ga += A[i * 3 + p] * A[i * 3 + q];
        }
        if (fabs(ga) <= 1e-300 || fabs(ga) <= 2.220446049250313e-16 * sqrt(al * be))
          continue;
        rotated = 1;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < 3; i++) {
          const double ap = A[i * 3 + p], aq = A[i * 3 + q];
          A[i * 3 + p] = c * ap - s * aq;
          A[i * 3 + q] = s * ap + c * aq;
          const double vp = Vm[i * 3 + p], vq = Vm[i * 3 + q];
          Vm[i * 3 + p] = c * vp - s * vq;
          Vm[i * 3 + q] = s * vp + c * vq;
        }
      }
    if (!rotated) break;
  }
  /* U = A Sigma^-1 column by column; a zero singular value gets the
   * orthonormal completion. */
  double U[9];
  double sig[3];
  for (int j = 0; j < 3; j++) {
    sig[j] = sqrt(A[j] * A[j] + A[3 + j] * A[3 + j] + A[6 + j] * A[6 + j]);
    for (int i = 0; i < 3; i++) U[i * 3 + j] = sig[j] > 0 ? A[i * 3 + j] / sig[j] : 0.0;
  }
  for (int j = 0; j < 3; j++)
    if (!(sig[j] > 0)) {
      const int a = (j + 1) % 3, b = (j + 2) % 3;
      U[0 * 3 + j] = U[1 * 3 + a] * U[2 * 3 + b] - U[2 * 3 + a] * U[1 * 3 + b];
      U[1 * 3 + j] = U[2 * 3 + a] * U[0 * 3 + b] - U[0 * 3 + a] * U[2 * 3 + b];
      U[2 * 3 + j] = U[0 * 3 + a] * U[1 * 3 + b] - U[1 * 3 + a] * U[0 * 3 + b];
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += U[i * 3 + k] * Vm[j * 3 + k];
      R[i * 3 + j] = s;
    }
}

/* RIGID projection: replace I+P by the orthogonal factor U V^T of its SVD.
 * RemoveTransformationScaling, broccoli_lib.cpp:6153-6194. */
void FN(orc_remove_scaling)(REAL* p) {
  double M[9], R[9];
  for (int i = 0; i < 9; i++) M[i] = (double)p[3 + i];
  M[0] += 1.0;
  M[4] += 1.0;
  M[8] += 1.0;
  FN(orc_polar3)(M, R);
  R[0] -= 1.0;
  R[4] -= 1.0;
  R[8] -= 1.0;
  for (int i = 0; i < 9; i++) p[3 + i] = (REAL)R[i];
}

/* 4x4 homogeneous matrix of a parameter vector; the diagonal one is added
 * in `real` before widening, as the reference does ((double)(p + 1.0f)). */
static void FN(orc_to_mat4)(const REAL* p, double tscale, double* Mt) {
  Mt[0] = (double)(p[3] + RONE); Mt[1] = (double)p[4]; Mt[2] = (double)p[5];
  Mt[3] = (double)(tscale == 1.0 ? p[0] : p[0] * (REAL)tscale);
  Mt[4] = (double)p[6]; Mt[5] = (double)(p[7] + RONE); Mt[6] = (double)p[8];
  Mt[7] = (double)(tscale == 1.0 ? p[1] : p[1] * (REAL)tscale);
  Mt[8] = (double)p[9]; Mt[9] = (double)p[10]; Mt[10] = (double)(p[11] + RONE);
  Mt[11] = (double)(tscale == 1.0 ? p[2] : p[2] * (REAL)tscale);
  Mt[12] = 0; Mt[13] = 0; Mt[14] = 0; Mt[15] = 1;
}

static void FN(orc_compose)(REAL* old12, const REAL* new12, double tscale) {
  double O[16], N[16], T[16];
  FN(orc_to_mat4)(old12, tscale, O);
  FN(orc_to_mat4)(new12, tscale, N);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += N[i * 4 + k] * O[k * 4 + j];
      T[i * 4 + j] = s;
    }
  old12[0] = (REAL)T[3];
  old12[1] = (REAL)T[7];
  old12[2] = (REAL)T[11];
  old12[3] = (REAL)(T[0] - 1.0); old12[4] = (REAL)T[1]; old12[5] = (REAL)T[2];
  old12[6] = (REAL)T[4]; old12[7] = (REAL)(T[5] - 1.0); old12[8] = (REAL)T[6];
  old12[9] = (REAL)T[8]; old12[10] = (REAL)T[9]; old12[11] = (REAL)(T[10] - 1.0);
}

/* Total = New * Old.  AddAffineRegistrationParameters,
 * broccoli_lib.cpp:7252-7340. */
void FN(orc_add_affine)(REAL* old12, const REAL* new12) {
  FN(orc_compose)(old12, new12, 1.0);
}

/* Same with both translations doubled (next pyramid scale).
 * AddAffineRegistrationParametersNextScale, broccoli_lib.cpp:7344-7431. */
void FN(orc_add_affine_next_scale)(REAL* old12, const REAL* new12) {
  FN(orc_compose)(old12, new12, 2.0);
}

/* Euler angles in degrees.  CalculateRotationAnglesFromRotationMatrix,
 * broccoli_lib.cpp:6199-6244. */
void FN(orc_rotation_angles)(const REAL* p, REAL* rot) {
  const double PI_ = 3.14159265358979323846;
  double m[9];
  for (int i = 0; i < 9; i++) m[i] = (double)p[3 + i];
  m[0] += 1.0;
  m[4] += 1.0;
  m[8] += 1.0;
  const double a1 = -atan2(m[5], m[8]) * 180.0 / PI_;
  const double c2 = sqrt(m[0] * m[0] + m[1] * m[1]);
  const double a2 = -atan2(-m[2], c2) * 180.0 / PI_;
  const double s1 = sin(a1 * PI_ / 180.0), c1 = cos(a1 * PI_ / 180.0);
  const double a3 = -atan2(s1 * m[6] - c1 * m[3], c1 * m[4] - s1 * m[7]) * 180.0 / PI_;
  rot[0] = (REAL)a1;
  rot[1] = (REAL)a2;
  rot[2] = (REAL)a3;
}

/* OpenCL 1.2 (section 8.2) linear filtering of a float image with
 * CLK_ADDRESS_CLAMP_TO_EDGE and unnormalised coordinates, exact weights:
 * i0 = floor(u - 0.5), a = frac(u - 0.5), indices clamped to the edge. */
static REAL FN(orc_sample_linear)(const REAL* T, int W, int H, int D, REAL u,
                                  REAL v, REAL w) {
  const REAL uu = u - RHALF, vv = v - RHALF, ww = w - RHALF;
  const REAL fu = RFLOOR(uu), fv = RFLOOR(vv), fw = RFLOOR(ww);
  const REAL a = uu - fu, b = vv - fv, c = ww - fw;
  int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
  int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
#define CLAMPI(q, n) q = q < 0 ? 0 : (q > n - 1 ? n - 1 : q)
  CLAMPI(i0, W); CLAMPI(i1, W); CLAMPI(j0, H); CLAMPI(j1, H); CLAMPI(k0, D); CLAMPI(k1, D);
#undef CLAMPI
#define TV(i, j, k) T[(i) + (long)(j) * W + (long)(k) * W * H]
  return (RONE - a) * (RONE - b) * (RONE - c) * TV(i0, j0, k0) +
         a * (RONE - b) * (RONE - c) * TV(i1, j0, k0) +
         (RONE - a) * b * (RONE - c) * TV(i0, j1, k0) +
         a * b * (RONE - c) * TV(i1, j1, k0) +
         (RONE - a) * (RONE - b) * c * TV(i0, j0, k1) +
         a * (RONE - b) * c * TV(i1, j0, k1) +
         (RONE - a) * b * c * TV(i0, j1, k1) + a * b * c * TV(i1, j1, k1);
#undef TV
}

/* OpenCL 1.2 (section 8.2) nearest filtering with CLK_ADDRESS_CLAMP_TO_EDGE
 * and unnormalised coordinates: i = floor(u), clamped to the edge. */
static REAL FN(orc_sample_nearest)(const REAL* T, int W, int H, int D, REAL u,
                                   REAL v, REAL w) {
  int i = (int)RFLOOR(u), j = (int)RFLOOR(v), k = (int)RFLOOR(w);
  i = i < 0 ? 0 : (i > W - 1 ? W - 1 : i);
  j = j < 0 ? 0 : (j > H - 1 ? H - 1 : j);
  k = k < 0 ? 0 : (k > D - 1 ? D - 1 : k);
  return T[i + (long)j * W + (long)k * W * H];
}

/* Sample with INTERPOLATION_MODE 0 (NEAREST) or 1 (LINEAR). */
static REAL FN(orc_sample)(int interp, const REAL* T, int W, int H, int D, REAL u,
                           REAL v, REAL w) {
  return interp == 0 ? FN(orc_sample_nearest)(T, W, H, D, u, v, w)
                     : FN(orc_sample_linear)(T, W, H, D, u, v, w);
}

/* Affine warp: out(x) = linear sample of src at
 * x + t + (A - I)(x - c), c the volume centre.
 * InterpolateVolumeLinearLinear, kernelRegistration.cpp:1066-1101. */
void FN(orc_warp_affine)(const REAL* src, int W, int H, int D, const REAL* p,
                         REAL* out) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const REAL xf = (REAL)x - ((REAL)W - RONE) * RHALF;
        const REAL yf = (REAL)y - ((REAL)H - RONE) * RHALF;
        const REAL zf = (REAL)z - ((REAL)D - RONE) * RHALF;
        const REAL u = (REAL)x + p[0] + p[3] * xf + p[4] * yf + p[5] * zf + RHALF;
        const REAL v = (REAL)y + p[1] + p[6] * xf + p[7] * yf + p[8] * zf + RHALF;
        const REAL w = (REAL)z + p[2] + p[9] * xf + p[10] * yf + p[11] * zf + RHALF;
        out[x + (long)y * W + (long)z * W * H] = FN(orc_sample_linear)(src, W, H, D, u, v, w);
      }
}

/* Displacement-field warp.  InterpolateVolumeLinearNonLinear,
 * kernelRegistration.cpp:1111-1140. */
void FN(orc_warp_field)(const REAL* src, int W, int H, int D, const REAL* dx,
                        const REAL* dy, const REAL* dz, REAL* out) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const long i = x + (long)y * W + (long)z * W * H;
        const REAL u = (REAL)x + dx[i] + RHALF;
        const REAL v = (REAL)y + dy[i] + RHALF;
        const REAL w = (REAL)z + dz[i] + RHALF;
        out[i] = FN(orc_sample_linear)(src, W, H, D, u, v, w);
      }
}

/* One parameter vector applied to T consecutive volumes with NEAREST (0) or
 * LINEAR (1) interpolation.  TransformVolumesLinear, broccoli_lib.cpp:
 * 8267-8359 (InterpolateVolumeNearestLinear / LinearLinear,
 * kernelRegistration.cpp:995-1031, :1066-1101). */
void FN(orc_transform_affine)(const REAL* src, int W, int H, int D, int T, const REAL* p, int interp,
                              REAL* out) {
  const long V = (long)W * H * D;
  for (int t = 0; t < T; t++) {
    const REAL* s = src + t * V;
    REAL* o = out + t * V;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < D; z++)
      for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
          const REAL xf = (REAL)x - ((REAL)W - RONE) * RHALF;
          const REAL yf = (REAL)y - ((REAL)H - RONE) * RHALF;
          const REAL zf = (REAL)z - ((REAL)D - RONE) * RHALF;
          const REAL u = (REAL)x + p[0] + p[3] * xf + p[4] * yf + p[5] * zf + RHALF;
          const REAL v = (REAL)y + p[1] + p[6] * xf + p[7] * yf + p[8] * zf + RHALF;
          const REAL w = (REAL)z + p[2] + p[9] * xf + p[10] * yf + p[11] * zf + RHALF;
          o[x + (long)y * W + (long)z * W * H] = FN(orc_sample)(interp, s, W, H, D, u, v, w);
        }
  }
}

/* One displacement field applied to T consecutive volumes.
 * TransformVolumesNonLinear, broccoli_lib.cpp:8361-8451
 * (InterpolateVolumeNearestNonLinear / LinearNonLinear,
 * kernelRegistration.cpp:1032-1061, :1111-1140). */
void FN(orc_transform_field)(const REAL* src, int W, int H, int D, int T, const REAL* dx,
                             const REAL* dy, const REAL* dz, int interp, REAL* out) {
  const long V = (long)W * H * D;
  for (int t = 0; t < T; t++) {
    const REAL* s = src + t * V;
    REAL* o = out + t * V;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < D; z++)
      for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
          const long i = x + (long)y * W + (long)z * W * H;
          o[i] = FN(orc_sample)(interp, s, W, H, D, (REAL)x + dx[i] + RHALF, (REAL)y + dy[i] + RHALF,
                                (REAL)z + dz[i] + RHALF);
        }
  }
}

/* Linear registration of `aligned` (warped from `original`) to `ref` over a
 * fixed number of iterations.  AlignTwoVolumesLinear,
 * broccoli_lib.cpp:5273-5437: the reference is filtered once per call, each
 * iteration filters the current aligned volume, builds and solves the
 * normal equations, applies the TRANSLATION / RIGID / AFFINE update
 * (:5398-5421) and re-warps the original with the total parameters.  On
 * return `aligned` holds the last warp, p12 the total parameters and rot3
 * (RIGID only) the Euler angles in degrees. */
void FN(orc_align_linear)(const REAL* ref, REAL* aligned, const REAL* original,
                          int W, int H, int D, const REAL* filters, int niter,
                          int type, REAL* p12, REAL* rot3) {
  FN(orc_align_linear_cs)(ref, aligned, original, W, H, D, filters, niter, type, 0.0, p12, rot3);
}

/* orc_align_linear with the certainties smoothed by the separable 3x3x3
 * Gaussian of orc_normal_equations_smoothcert when cert_sigma > 0 (the
 * certainty-smoothing switch of the batched motion-correction workload;
 * not in the reference). */
void FN(orc_align_linear_cs)(const REAL* ref, REAL* aligned, const REAL* original,
                             int W, int H, int D, const REAL* filters, int niter,
                             int type, double cert_sigma, REAL* p12, REAL* rot3) {
  const long V = (long)W * H * D;
  REAL* q1 = (REAL*)malloc(sizeof(REAL) * 6 * V);
  REAL* q2 = (REAL*)malloc(sizeof(REAL) * 6 * V);
  REAL A[144], h[12], p[12];
  FN(orc_filter3d)(ref, W, H, D, filters, 3, q1);
  for (int i = 0; i < 12; i++) p12[i] = RZERO;
  for (int it = 0; it < niter; it++) {
    FN(orc_filter3d)(aligned, W, H, D, filters, 3, q2);
    if (cert_sigma > 0.0)
      FN(orc_normal_equations_smoothcert)(q1, q2, W, H, D, cert_sigma, A, h);
    else
      FN(orc_normal_equations)(q1, q2, W, H, D, A, h);
    FN(orc_solve)(A, h, 12, p);
    if (type == ORC_TRANSLATION) {
      p12[0] += p[0];
      p12[1] += p[1];
      p12[2] += p[2];
      for (int i = 3; i < 12; i++) p12[i] = RZERO;
    } else if (type == ORC_RIGID) {
      FN(orc_remove_scaling)(p);
      FN(orc_add_affine)(p12, p);
    } else {
      FN(orc_add_affine)(p12, p);
    }
    FN(orc_warp_affine)(original, W, H, D, p12, aligned);
  }
  if (type == ORC_RIGID && rot3) FN(orc_rotation_angles)(p12, rot3);
  free(q1);
  free(q2);
}

/* Rigid motion correction of a series to its first volume.
 * PerformMotionCorrectionWrapper, broccoli_lib.cpp:10658-10720: volume 0 is
 * the reference and keeps zero motion; every later volume is registered
 * (RIGID, niter iterations), replaced in place by its corrected copy, and
 * its motion is written as motion6T[t + k*T] for k = translations x,y,z in
 * mm (voxels times voxel size) then rotations in degrees. */
void FN(orc_motion_correct)(REAL* vols, int W, int H, int D, int T,
                            const REAL* voxel_size, const REAL* filters,
                            int niter, REAL* motion6T) {
  const long V = (long)W * H * D;
  REAL* ref = (REAL*)malloc(sizeof(REAL) * V);
  REAL* orig = (REAL*)malloc(sizeof(REAL) * V);
  for (long i = 0; i < V; i++) ref[i] = vols[i];
  for (int k = 0; k < 6; k++) motion6T[k * T] = RZERO;
  for (int t = 1; t < T; t++) {
    REAL p[12], rot[3];
    REAL* vt = vols + (long)t * V;
    for (long i = 0; i < V; i++) orig[i] = vt[i];
    FN(orc_align_linear)(ref, vt, orig, W, H, D, filters, niter, ORC_RIGID, p, rot);
    motion6T[t + 0 * T] = p[0] * voxel_size[0];
    motion6T[t + 1 * T] = p[1] * voxel_size[1];
    motion6T[t + 2 * T] = p[2] * voxel_size[2];
    motion6T[t + 3 * T] = rot[0];
    motion6T[t + 4 * T] = rot[1];
    motion6T[t + 5 * T] = rot[2];
  }
  free(ref);
  free(orig);
}

/* Gaussian smoothing filter of `size` taps for a given sigma (voxels),
 * normalised by its float sum.  CreateSmoothingFilters(..., double sigma),
 * broccoli_lib.cpp:11093-11121. */
void FN(orc_smoothing_filter_sigma)(int size, double sigma, REAL* f) {
  const int half = (size - 1) / 2;
  const double s2 = 2.0 * sigma * sigma;
  REAL sum = RZERO;
  for (int i = 0; i < size; i++) {
    const double u = (double)(i - half);
    f[i] = (REAL)exp(-pow(u, 2.0) / s2);
    sum += f[i];
  }
  for (int i = 0; i < size; i++) f[i] /= sum;
}

/* Per-axis Gaussian filters from a FWHM in mm and the voxel sizes.
 * CreateSmoothingFilters(..., FWHM, voxel sizes), broccoli_lib.cpp:11055-11091. */
void FN(orc_smoothing_filter_fwhm)(int size, double fwhm, double vx, double vy,
                                   double vz, REAL* fx, REAL* fy, REAL* fz) {
  const int half = (size - 1) / 2;
  const double sx = fwhm / 2.354 / vx, sy = fwhm / 2.354 / vy, sz = fwhm / 2.354 / vz;
  const double sx2 = 2.0 * sx * sx, sy2 = 2.0 * sy * sy, sz2 = 2.0 * sz * sz;
  REAL ax = RZERO, ay = RZERO, az = RZERO;
  for (int i = 0; i < size; i++) {
    const double u = (double)(i - half);
    fx[i] = (REAL)exp(-pow(u, 2.0) / sx2);
    fy[i] = (REAL)exp(-pow(u, 2.0) / sy2);
    fz[i] = (REAL)exp(-pow(u, 2.0) / sz2);
    ax += fx[i];
    ay += fy[i];
    az += fz[i];
  }
  for (int i = 0; i < size; i++) {
    fx[i] /= ax;
    fy[i] /= ay;
    fz[i] /= az;
  }
}

/* Separable 9-tap normalised convolution: along y of vol*cert (Rows,
 * kernelConvolution.cpp:52-91), along x (Columns, :531-569), along z divided
 * by the smoothed certainty (Rods, :1201-1240).  Zero padding; the filter
 * index runs 8..0 as the offset runs -4..+4.  cert / smoothed_cert may be
 * NULL for all-ones (the in-place smoothing of PerformSmoothing,
 * broccoli_lib.cpp:11274-11357 and :11461-11545). */
void FN(orc_smooth3d)(const REAL* vol, const REAL* cert, const REAL* scert,
                      int W, int H, int D, const REAL* fx, const REAL* fy,
                      const REAL* fz, REAL* out) {
  const long V = (long)W * H * D;
  REAL* rows = (REAL*)malloc(sizeof(REAL) * V);
  REAL* cols = (REAL*)malloc(sizeof(REAL) * V);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        REAL s = RZERO;
        int off = -4;
        for (int f = 8; f >= 0; f--, off++) {
          REAL px = RZERO;
          if (y + off >= 0 && y + off < H) {
            const long j = x + (long)(y + off) * W + (long)z * W * H;
            px = cert ? vol[j] * cert[j] : vol[j] * RONE;
          }
          s += px * fy[f];
        }
        rows[x + (long)y * W + (long)z * W * H] = s;
      }
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        REAL s = RZERO;
        int off = -4;
        for (int f = 8; f >= 0; f--, off++) {
          REAL px = RZERO;
          if (x + off >= 0 && x + off < W) px = rows[x + off + (long)y * W + (long)z * W * H];
          s += px * fx[f];
        }
        cols[x + (long)y * W + (long)z * W * H] = s;
      }
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        REAL s = RZERO;
        int off = -4;
        for (int f = 8; f >= 0; f--, off++) {
          REAL px = RZERO;
          if (z + off >= 0 && z + off < D) px = cols[x + (long)y * W + (long)(z + off) * W * H];
          s += px * fz[f];
        }
        const long i = x + (long)y * W + (long)z * W * H;
        out[i] = s / (scert ? scert[i] : RONE);
      }
  free(rows);
  free(cols);
}

/* Resample to a new grid size by linear interpolation with sample spacing
 * (N-1)/(N'-1) per axis.  RescaleVolumeLinear, kernelRegistration.cpp:
 * 1340-1366, driven by ChangeVolumeSize, broccoli_lib.cpp:6247-6388. */
static void FN(orc_rescale_interp)(const REAL* src, int W, int H, int D, int W2,
                                   int H2, int D2, int interp, REAL* out) {
  const REAL dx = (REAL)(W - 1) / (REAL)(W2 - 1);
  const REAL dy = (REAL)(H - 1) / (REAL)(H2 - 1);
  const REAL dz = (REAL)(D - 1) / (REAL)(D2 - 1);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D2; z++)
    for (int y = 0; y < H2; y++)
      for (int x = 0; x < W2; x++)
        out[x + (long)y * W2 + (long)z * W2 * H2] = FN(orc_sample)(
            interp, src, W, H, D, (REAL)x * dx + RHALF, (REAL)y * dy + RHALF, (REAL)z * dz + RHALF);
}

void FN(orc_rescale_linear)(const REAL* src, int W, int H, int D, int W2,
                            int H2, int D2, REAL* out) {
  FN(orc_rescale_interp)(src, W, H, D, W2, H2, D2, 1, out);
}

/* myround, broccoli_lib.cpp:94-97. */
static int FN(orc_myround)(float a) { return (int)floorf(a + 0.5f); }

/* Multi-scale linear registration.  AlignTwoVolumesLinearSeveralScales,
 * broccoli_lib.cpp:6391-6513: both volumes are resampled to
 * round(N/scale) per axis; at every scale after the coarsest the resampled
 * moving volume is first warped with the total parameters found so far and
 * that warped copy is what the scale registers; the coarse-scale totals are
 * carried to the next scale with doubled translations
 * (AddAffineRegistrationParametersNextScale); the finest scale runs
 * ceil(niter/5) iterations; the rotations of all scales are summed.  On
 * return `aligned` (full size) is the moving volume warped by the total
 * parameters (the DO_OVERWRITE behaviour). */
void FN(orc_align_linear_scales)(const REAL* ref, REAL* aligned, int W, int H, int D,
                                 int coarsest, const REAL* filters, int niter, int type,
                                 REAL* p12, REAL* rot3) {
  const long V = (long)W * H * D;
  REAL* orig_full = (REAL*)malloc(sizeof(REAL) * V);
  for (long i = 0; i < V; i++) orig_full[i] = aligned[i];
  REAL tmp[12], rt[3] = {RZERO, RZERO, RZERO};
  for (int i = 0; i < 12; i++) p12[i] = RZERO;
  if (rot3) rot3[0] = rot3[1] = rot3[2] = RZERO;
  int cw = FN(orc_myround)((float)W / (float)coarsest);
  int ch = FN(orc_myround)((float)H / (float)coarsest);
  int cd = FN(orc_myround)((float)D / (float)coarsest);
  REAL* r_s = (REAL*)malloc(sizeof(REAL) * V);
  REAL* o_s = (REAL*)malloc(sizeof(REAL) * V);
  REAL* a_s = (REAL*)malloc(sizeof(REAL) * V);
  FN(orc_rescale_linear)(orig_full, W, H, D, cw, ch, cd, o_s);
  FN(orc_rescale_linear)(ref, W, H, D, cw, ch, cd, r_s);
  for (int scale = coarsest; scale >= 1; scale /= 2) {
    const long vs = (long)cw * ch * cd;
    for (long i = 0; i < vs; i++) a_s[i] = o_s[i];
    const int it = scale == 1 ? (int)ceilf((float)niter / 5.0f) : niter;
    FN(orc_align_linear)(r_s, a_s, o_s, cw, ch, cd, filters, it, type, tmp, rt);
    if (type != ORC_RIGID) rt[0] = rt[1] = rt[2] = RZERO;
    if (scale != 1) {
      if (rot3) {
        rot3[0] += rt[0];
        rot3[1] += rt[1];
        rot3[2] += rt[2];
      }
      FN(orc_add_affine_next_scale)(p12, tmp);
      cw = FN(orc_myround)((float)W / ((float)scale / 2.0f));
      ch = FN(orc_myround)((float)H / ((float)scale / 2.0f));
      cd = FN(orc_myround)((float)D / ((float)scale / 2.0f));
      REAL* resc = (REAL*)malloc(sizeof(REAL) * (long)cw * ch * cd);
      FN(orc_rescale_linear)(orig_full, W, H, D, cw, ch, cd, resc);
      FN(orc_rescale_linear)(ref, W, H, D, cw, ch, cd, r_s);
      FN(orc_warp_affine)(resc, cw, ch, cd, p12, o_s);
      free(resc);
    } else {
      FN(orc_add_affine)(p12, tmp);
      if (rot3) {
        rot3[0] += rt[0];
        rot3[1] += rt[1];
        rot3[2] += rt[2];
      }
      FN(orc_warp_affine)(orig_full, W, H, D, p12, aligned);
    }
  }
  free(orig_full);
  free(r_s);
  free(o_s);
  free(a_s);
}

/* Structure tensor of the aligned volume: T = sum_k |q2_k| M_k, with M_k
 * the projection tensor (m11 m12 m13 m22 m23 m33) of filter k.
 * CalculateTensorComponents, kernelRegistration.cpp:806-845 (called once
 * per filter, accumulating). */
void FN(orc_tensor_components)(const REAL* q2, long V, const REAL* m6, REAL* t6) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < V; i++) {
    const REAL mag = RSQRT(q2[2 * i] * q2[2 * i] + q2[2 * i + 1] * q2[2 * i + 1]);
    for (int c = 0; c < 6; c++) t6[(long)c * V + i] += mag * m6[c];
  }
}

/* Frobenius norm of the symmetric tensor.  CalculateTensorNorms,
 * kernelRegistration.cpp:847-875. */
void FN(orc_tensor_norms)(const REAL* t6, long V, REAL* norm) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < V; i++) {
    const REAL a = t6[i], b = t6[V + i], c = t6[2 * V + i], d = t6[3 * V + i],
               e = t6[4 * V + i], f = t6[5 * V + i];
    norm[i] = RSQRT(a * a + (REAL)2.0 * b * b + (REAL)2.0 * c * c + d * d + (REAL)2.0 * e * e + f * f);
  }
}

/* a += c TT and h += c dphi TT n for one filter, with TT = T T (symmetric)
 * and c = sqrt|q1 q2*| cos^2(dphi/2).  CalculateAMatricesAndHVectors,
 * kernelRegistration.cpp:880-943.  a6: a11 a12 a13 a22 a23 a33; h3. */
void FN(orc_nonlinear_ah)(const REAL* q1, const REAL* q2, const REAL* t6, long V, REAL nx, REAL ny,
                          REAL nz, REAL* a6, REAL* h3) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < V; i++) {
    const REAL q1x = q1[2 * i], q1y = q1[2 * i + 1], q2x = q2[2 * i], q2y = q2[2 * i + 1];
    const REAL qr = q1x * q2x + q1y * q2y;
    const REAL qi = -q1x * q2y + q1y * q2x;
    const REAL pd = RATAN2(qi, qr);
    const REAL aqq = RSQRT(qr * qr + qi * qi);
    const REAL cert = RSQRT(aqq) * RCOS(pd / (REAL)2.0) * RCOS(pd / (REAL)2.0);
    const REAL t11 = t6[i], t12 = t6[V + i], t13 = t6[2 * V + i], t22 = t6[3 * V + i],
               t23 = t6[4 * V + i], t33 = t6[5 * V + i];
    const REAL tt11 = t11 * t11 + t12 * t12 + t13 * t13;
    const REAL tt12 = t11 * t12 + t12 * t22 + t13 * t23;
    const REAL tt13 = t11 * t13 + t12 * t23 + t13 * t33;
    const REAL tt22 = t12 * t12 + t22 * t22 + t23 * t23;
    const REAL tt23 = t12 * t13 + t22 * t23 + t23 * t33;
    const REAL tt33 = t13 * t13 + t23 * t23 + t33 * t33;
    a6[i] += cert * tt11;
    a6[V + i] += cert * tt12;
    a6[2 * V + i] += cert * tt13;
    a6[3 * V + i] += cert * tt22;
    a6[4 * V + i] += cert * tt23;
    a6[5 * V + i] += cert * tt33;
    h3[i] += cert * pd * (nx * tt11 + ny * tt12 + nz * tt13);
    h3[V + i] += cert * pd * (nx * tt12 + ny * tt22 + nz * tt23);
    h3[2 * V + i] += cert * pd * (nx * tt13 + ny * tt23 + nz * tt33);
  }
}

/* Per-voxel 3x3 solve by cofactors with det + 1e-16.
 * CalculateDisplacementUpdate, kernelRegistration.cpp:948-988. */
void FN(orc_displacement_update)(const REAL* a6, const REAL* h3, long V, REAL* d3) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < V; i++) {
    const REAL a11 = a6[i], a12 = a6[V + i], a13 = a6[2 * V + i], a22 = a6[3 * V + i],
               a23 = a6[4 * V + i], a33 = a6[5 * V + i];
    const REAL h1 = h3[i], h2 = h3[V + i], hh3 = h3[2 * V + i];
    const REAL norm = RONE / (a11 * a22 * a33 - a11 * a23 * a23 - a12 * a12 * a33 + a12 * a23 * a13 +
                              a13 * a12 * a23 - a13 * a22 * a13 + (REAL)1e-16);
    d3[i] = norm * ((hh3 * (a12 * a23 - a13 * a22)) - (h2 * (a12 * a33 - a13 * a23)) +
                    (h1 * (a22 * a33 - a23 * a23)));
    d3[V + i] = norm * ((h2 * (a11 * a33 - a13 * a13)) - (hh3 * (a11 * a23 - a13 * a12)) -
                        (h1 * (a12 * a33 - a23 * a13)));
    d3[2 * V + i] = norm * ((hh3 * (a11 * a22 - a12 * a12)) - (h2 * (a11 * a23 - a12 * a13)) +
                            (h1 * (a12 * a23 - a22 * a13)));
  }
}

/* Nonlinear (displacement field) registration at one scale.
 * AlignTwoVolumesNonLinear, broccoli_lib.cpp:5748-6058.  Per iteration:
 * six responses of the aligned volume; structure tensor from their
 * magnitudes; tensor smoothed (tsigma); tensor norm written into a11 (it
 * stays there: a11 = norm + sum c tt11, the reference's accumulation); the
 * tensor is divided by its largest norm (max from FLT_MIN); A and h from
 * the six filter pairs; A, h smoothed (esigma); 3x3 solve per voxel;
 * update smoothed (dsigma) and added to the field; the original re-warped
 * by the field.  tensors: 6 x {m11 m12 m13 m22 m23 m33}; dirs: x[6] y[6]
 * z[6]; field: 3 volumes (x, y, z), zeroed here. */
void FN(orc_align_nonlinear)(const REAL* ref, REAL* aligned, const REAL* original, int W, int H,
                             int D, const REAL* filters6, const REAL* tensors, const REAL* dirs,
                             int niter, double tsigma, double esigma, double dsigma, REAL* field) {
  const long V = (long)W * H * D;
  REAL* q1 = (REAL*)malloc(sizeof(REAL) * 12 * V);
  REAL* q2 = (REAL*)malloc(sizeof(REAL) * 12 * V);
  REAL* t6 = (REAL*)malloc(sizeof(REAL) * 6 * V);
  REAL* a6 = (REAL*)malloc(sizeof(REAL) * 6 * V);
  REAL* h3 = (REAL*)malloc(sizeof(REAL) * 3 * V);
  REAL* d3 = (REAL*)malloc(sizeof(REAL) * 3 * V);
  REAL* tmp = (REAL*)malloc(sizeof(REAL) * V);
  REAL ft[9], fe[9], fd[9];
  FN(orc_smoothing_filter_sigma)(9, tsigma, ft);
  FN(orc_smoothing_filter_sigma)(9, esigma, fe);
  FN(orc_smoothing_filter_sigma)(9, dsigma, fd);
  FN(orc_filter3d)(ref, W, H, D, filters6, 6, q1);
  for (long i = 0; i < 3 * V; i++) field[i] = RZERO;
  for (int it = 0; it < niter; it++) {
    FN(orc_filter3d)(aligned, W, H, D, filters6, 6, q2);
    for (long i = 0; i < 6 * V; i++) t6[i] = RZERO;
    for (long i = 0; i < 6 * V; i++) a6[i] = RZERO;
    for (long i = 0; i < 3 * V; i++) h3[i] = RZERO;
    for (int k = 0; k < 6; k++) FN(orc_tensor_components)(q2 + (long)k * 2 * V, V, tensors + 6 * k, t6);
    for (int c = 0; c < 6; c++) {
      FN(orc_smooth3d)(t6 + (long)c * V, NULL, NULL, W, H, D, ft, ft, ft, tmp);
      for (long i = 0; i < V; i++) t6[(long)c * V + i] = tmp[i];
    }
    FN(orc_tensor_norms)(t6, V, a6);
    float mx = 1.17549435e-38f;
    for (long i = 0; i < V; i++) mx = (float)a6[i] > mx ? (float)a6[i] : mx;
    const REAL f = (REAL)(1.0f / mx);
    for (long i = 0; i < 6 * V; i++) t6[i] = t6[i] * f;
    for (int k = 0; k < 6; k++)
      FN(orc_nonlinear_ah)(q1 + (long)k * 2 * V, q2 + (long)k * 2 * V, t6, V, dirs[k], dirs[6 + k],
                           dirs[12 + k], a6, h3);
    for (int c = 0; c < 6; c++) {
      FN(orc_smooth3d)(a6 + (long)c * V, NULL, NULL, W, H, D, fe, fe, fe, tmp);
      for (long i = 0; i < V; i++) a6[(long)c * V + i] = tmp[i];
    }
    for (int c = 0; c < 3; c++) {
      FN(orc_smooth3d)(h3 + (long)c * V, NULL, NULL, W, H, D, fe, fe, fe, tmp);
      for (long i = 0; i < V; i++) h3[(long)c * V + i] = tmp[i];
    }
    FN(orc_displacement_update)(a6, h3, V, d3);
    for (int c = 0; c < 3; c++) {
      FN(orc_smooth3d)(d3 + (long)c * V, NULL, NULL, W, H, D, fd, fd, fd, tmp);
      for (long i = 0; i < V; i++) field[(long)c * V + i] = field[(long)c * V + i] + tmp[i];
    }
    FN(orc_warp_field)(original, W, H, D, field, field + V, field + 2 * V, aligned);
  }
  free(q1);
  free(q2);
  free(t6);
  free(a6);
  free(h3);
  free(d3);
  free(tmp);
}

/* Multi-scale nonlinear registration.  AlignTwoVolumesNonLinearSeveralScales,
 * broccoli_lib.cpp:6516-6665: scales coarsest..1 (halving); each scale
 * registers the resampled moving volume pre-warped by the total field so far
 * (resampled to the scale and doubled, :6604-6611); the finest scale runs
 * ceil(niter/2) iterations.  On return `field` (3 full-size volumes) is the
 * total field and `aligned` the moving volume warped by it. */
void FN(orc_align_nonlinear_scales)(const REAL* ref, REAL* aligned, int W, int H, int D,
                                    int coarsest, const REAL* filters6, const REAL* tensors,
                                    const REAL* dirs, int niter, double tsigma, double esigma,
                                    double dsigma, REAL* field) {
  const long V = (long)W * H * D;
  REAL* orig_full = (REAL*)malloc(sizeof(REAL) * V);
  for (long i = 0; i < V; i++) orig_full[i] = aligned[i];
  int cw = FN(orc_myround)((float)W / (float)coarsest);
  int ch = FN(orc_myround)((float)H / (float)coarsest);
  int cd = FN(orc_myround)((float)D / (float)coarsest);
  REAL* r_s = (REAL*)malloc(sizeof(REAL) * V);
  REAL* o_s = (REAL*)malloc(sizeof(REAL) * V);
  REAL* a_s = (REAL*)malloc(sizeof(REAL) * V);
  REAL* tot = (REAL*)calloc(3 * V, sizeof(REAL));
  REAL* upd = (REAL*)malloc(sizeof(REAL) * 3 * V);
  REAL* tmp = (REAL*)malloc(sizeof(REAL) * 3 * V);
  FN(orc_rescale_linear)(orig_full, W, H, D, cw, ch, cd, o_s);
  FN(orc_rescale_linear)(ref, W, H, D, cw, ch, cd, r_s);
  for (int scale = coarsest; scale >= 1; scale /= 2) {
    const long vs = (long)cw * ch * cd;
    for (long i = 0; i < vs; i++) a_s[i] = o_s[i];
    const int it = scale == 1 ? (int)ceilf((float)niter / 2.0f) : niter;
    FN(orc_align_nonlinear)(r_s, a_s, o_s, cw, ch, cd, filters6, tensors, dirs, it, tsigma, esigma,
                            dsigma, upd);
    for (int c = 0; c < 3; c++)
      for (long i = 0; i < vs; i++) tot[c * vs + i] = tot[c * vs + i] + upd[c * vs + i];
    if (scale != 1) {
      const int pw = cw, ph = ch, pdp = cd;
      cw = FN(orc_myround)((float)W / ((float)scale / 2.0f));
      ch = FN(orc_myround)((float)H / ((float)scale / 2.0f));
      cd = FN(orc_myround)((float)D / ((float)scale / 2.0f));
      const long nv = (long)cw * ch * cd;
      for (int c = 0; c < 3; c++) FN(orc_rescale_linear)(tot + c * (long)pw * ph * pdp, pw, ph, pdp, cw, ch, cd, tmp + c * nv);
      for (long i = 0; i < 3 * nv; i++) tot[i] = tmp[i] * (REAL)2.0;
      REAL* resc = (REAL*)malloc(sizeof(REAL) * nv);
      FN(orc_rescale_linear)(orig_full, W, H, D, cw, ch, cd, resc);
      FN(orc_rescale_linear)(ref, W, H, D, cw, ch, cd, r_s);
      FN(orc_warp_field)(resc, cw, ch, cd, tot, tot + nv, tot + 2 * nv, o_s);
      free(resc);
    } else {
      for (long i = 0; i < 3 * V; i++) field[i] = tot[i];
      FN(orc_warp_field)(orig_full, W, H, D, field, field + V, field + 2 * V, aligned);
    }
  }
  free(orig_full);
  free(r_s);
  free(o_s);
  free(a_s);
  free(tot);
  free(upd);
  free(tmp);
}

/* Resample a volume to new voxel sizes, then centre it in (or crop it to)
 * the new grid, with an extra shift of mm_z_cut mm along z.
 * ChangeVolumesResolutionAndSize, broccoli_lib.cpp:6950-7100, with
 * RescaleVolumeLinear and CopyVolumeToNew (kernelRegistration.cpp:
 * 1340-1366, :1593-1678).  Voxels of the new grid not covered stay 0. */
void FN(orc_change_resolution_and_size_interp)(const REAL* src, int W, int H, int D, float vx,
                                               float vy, float vz, REAL* out, int W2, int H2, int D2,
                                               float nvx, float nvy, float nvz, int mm_z_cut,
                                               int mode) {
  const int Wi = FN(orc_myround)((float)W * vx / nvx);
  const int Hi = FN(orc_myround)((float)H * vy / nvy);
  const int Di = FN(orc_myround)((float)D * vz / nvz);
  REAL* interp = (REAL*)malloc(sizeof(REAL) * (long)Wi * Hi * Di);
  FN(orc_rescale_interp)(src, W, H, D, Wi, Hi, Di, mode, interp);
  for (long i = 0; i < (long)W2 * H2 * D2; i++) out[i] = RZERO;
  const int xd = Wi - W2, yd = Hi - H2, zd = Di - D2;
  const int zcut = (int)round((float)mm_z_cut / nvz);
  const int gx = W2 > Wi ? W2 : Wi, gy = H2 > Hi ? H2 : Hi, gz = D2 > Di ? D2 : Di;
  for (int z = 0; z < gz; z++)
    for (int y = 0; y < gy; y++)
      for (int x = 0; x < gx; x++) {
        int xn, xi, yn, yi, zn, zi;
        if (xd > 0) { xn = x; xi = x + (int)round((float)xd / 2.0); }
        else { xn = x + (int)round((float)abs(xd) / 2.0); xi = x; }
        if (yd > 0) { yn = y; yi = y + (int)round((float)yd / 2.0); }
        else { yn = y + (int)round((float)abs(yd) / 2.0); yi = y; }
        if (zd > 0) { zn = z; zi = z + (int)round((float)zd / 2.0) + zcut; }
        else { zn = z + (int)round((float)abs(zd) / 2.0); zi = z + zcut; }
        if (xi >= Wi || yi >= Hi || zi >= Di || xn >= W2 || yn >= H2 || zn >= D2) continue;
        if (xi < 0 || yi < 0 || zi < 0 || xn < 0 || yn < 0 || zn < 0) continue;
        out[xn + (long)yn * W2 + (long)zn * W2 * H2] = interp[xi + (long)yi * Wi + (long)zi * Wi * Hi];
      }
  free(interp);
}

void FN(orc_change_resolution_and_size)(const REAL* src, int W, int H, int D, float vx, float vy,
                                        float vz, REAL* out, int W2, int H2, int D2, float nvx,
                                        float nvy, float nvz, int mm_z_cut) {
  FN(orc_change_resolution_and_size_interp)(src, W, H, D, vx, vy, vz, out, W2, H2, D2, nvx, nvy, nvz,
                                            mm_z_cut, 1);
}

/* Centre of mass (voxels), float accumulation in x-fastest order.
 * CalculateCenterOfMass, broccoli_lib.cpp:6763-6800. */
void FN(orc_center_of_mass)(const REAL* vol, int W, int H, int D, REAL* c3) {
  REAL tm = RZERO, rx = RZERO, ry = RZERO, rz = RZERO;
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const REAL m = vol[x + (long)y * W + (long)z * W * H];
        rx += m * (REAL)x;
        ry += m * (REAL)y;
        rz += m * (REAL)z;
        tm += m;
      }
  c3[0] = rx / tm;
  c3[1] = ry / tm;
  c3[2] = rz / tm;
}

/* Centre T volumes by the centre of mass of the first: the integer
 * translation -myround(N/2 - com) per axis, applied to all T volumes with
 * the given interpolation.  CenterVolumesWrapper / CenterVolumeMass,
 * broccoli_lib.cpp:6839-6874, :8225-8245. */
void FN(orc_center_volumes)(const REAL* src, int W, int H, int D, int T, int interp, REAL* out,
                            REAL* p12) {
  REAL c[3];
  FN(orc_center_of_mass)(src, W, H, D, c);
  for (int i = 0; i < 12; i++) p12[i] = RZERO;
  p12[0] = -(REAL)FN(orc_myround)((float)W / 2.0f - (float)c[0]);
  p12[1] = -(REAL)FN(orc_myround)((float)H / 2.0f - (float)c[1]);
  p12[2] = -(REAL)FN(orc_myround)((float)D / 2.0f - (float)c[2]);
  FN(orc_transform_affine)(src, W, H, D, T, p12, interp, out);
}

/* Translate v1 by the rounded difference of the centres of mass so that it
 * overlaps v2; returns the translation as parameters.
 * MatchVolumeMasses, broccoli_lib.cpp:6876-6948. */
void FN(orc_match_volume_masses)(REAL* v1, const REAL* v2, int W, int H, int D, REAL* p12) {
  REAL c1[3], c2[3];
  FN(orc_center_of_mass)(v1, W, H, D, c1);
  FN(orc_center_of_mass)(v2, W, H, D, c2);
  for (int i = 0; i < 12; i++) p12[i] = RZERO;
  p12[0] = -(REAL)FN(orc_myround)((float)(c2[0] - c1[0]));
  p12[1] = -(REAL)FN(orc_myround)((float)(c2[1] - c1[1]));
  p12[2] = -(REAL)FN(orc_myround)((float)(c2[2] - c1[2]));
  const long V = (long)W * H * D;
  REAL* tmp = (REAL*)malloc(sizeof(REAL) * V);
  for (long i = 0; i < V; i++) tmp[i] = v1[i];
  FN(orc_warp_affine)(tmp, W, H, D, p12, v1);
  free(tmp);
}

/* field += affine displacement t + (A - I)(x - c).
 * AddLinearAndNonLinearDisplacement, kernelRegistration.cpp:1142-1178. */
void FN(orc_add_linear_nonlinear)(REAL* field, int W, int H, int D, const REAL* p) {
  const long V = (long)W * H * D;
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const REAL xf = (REAL)x - ((REAL)W - RONE) * RHALF;
        const REAL yf = (REAL)y - ((REAL)H - RONE) * RHALF;
        const REAL zf = (REAL)z - ((REAL)D - RONE) * RHALF;
        const long i = x + (long)y * W + (long)z * W * H;
        field[i] += p[0] + p[3] * xf + p[4] * yf + p[5] * zf;
        field[V + i] += p[1] + p[6] * xf + p[7] * yf + p[8] * zf;
        field[2 * V + i] += p[2] + p[9] * xf + p[10] * yf + p[11] * zf;
      }
}

/* T1-to-template normalisation.  PerformRegistrationTwoVolumesWrapper,
 * broccoli_lib.cpp:7973-8112 (single volume, no pre-centring, no skull
 * strip): resample the input onto the template grid; match centres of
 * mass; multi-scale AFFINE registration; parameters composed with the mass
 * match; multi-scale nonlinear registration; the affine motion added to the
 * field; the input resampled again and warped once by the combined field.
 * Outputs (template size): params12, interpolated (after the resample and
 * mass match), aligned_linear, aligned_nonlinear and field (3 volumes). */
void FN(orc_register_two_volumes)(const REAL* in, int W, int H, int D, const float* vin,
                                  const REAL* tpl, int W2, int H2, int D2, const float* vtpl,
                                  int mm_z_cut, int coarsest, int lin_iter, int nl_iter,
                                  const REAL* filters3, const REAL* filters6, const REAL* tensors,
                                  const REAL* dirs, double tsigma, double esigma, double dsigma,
                                  REAL* p12, REAL* interpolated, REAL* aligned_linear,
                                  REAL* aligned_nonlinear, REAL* field) {
  const long V2 = (long)W2 * H2 * D2;
  REAL* work = (REAL*)malloc(sizeof(REAL) * V2);
  REAL match[12], rot[3];
  for (int i = 0; i < 12; i++) p12[i] = RZERO;
  FN(orc_change_resolution_and_size)(in, W, H, D, vin[0], vin[1], vin[2], work, W2, H2, D2, vtpl[0],
                                     vtpl[1], vtpl[2], mm_z_cut);
  FN(orc_match_volume_masses)(work, tpl, W2, H2, D2, match);
  for (long i = 0; i < V2; i++) interpolated[i] = work[i];
  FN(orc_align_linear_scales)(tpl, work, W2, H2, D2, coarsest, filters3, lin_iter, ORC_AFFINE, p12, rot);
  for (long i = 0; i < V2; i++) aligned_linear[i] = work[i];
  FN(orc_add_affine)(p12, match);
  FN(orc_align_nonlinear_scales)(tpl, work, W2, H2, D2, coarsest, filters6, tensors, dirs, nl_iter,
                                 tsigma, esigma, dsigma, field);
  FN(orc_add_linear_nonlinear)(field, W2, H2, D2, p12);
  FN(orc_change_resolution_and_size)(in, W, H, D, vin[0], vin[1], vin[2], work, W2, H2, D2, vtpl[0],
                                     vtpl[1], vtpl[2], mm_z_cut);
  FN(orc_warp_field)(work, W2, H2, D2, field, field + V2, field + 2 * V2, aligned_nonlinear);
  free(work);
}

/* Tensor magnitude of one volume: its six nonlinear filter responses, the
 * structure tensor T = sum_k |q_k| M_k and the Frobenius norm of T.
 * CalculateTensorMagnitude, broccoli_lib.cpp:5658-5746 (responses of the
 * volume in the q2 slots; CalculateTensorComponents,
 * kernelRegistration.cpp:806-845, reads only q2; CalculateTensorNorms,
 * :847-875). */
void FN(orc_tensor_magnitude)(const REAL* vol, int W, int H, int D, const REAL* filters6,
                              const REAL* tensors, REAL* out) {
  const long V = (long)W * H * D;
  REAL* q = (REAL*)malloc(sizeof(REAL) * 12 * V);
  REAL* t6 = (REAL*)calloc(6 * V, sizeof(REAL));
  FN(orc_filter3d)(vol, W, H, D, filters6, 6, q);
  for (int k = 0; k < 6; k++) FN(orc_tensor_components)(q + 2 * V * k, V, tensors + 6 * k, t6);
  FN(orc_tensor_norms)(t6, V, out);
  free(q);
  free(t6);
}

/* Brain mask of one EPI volume.  SegmentEPIData, broccoli_lib.cpp:
 * 11008-11030: smoothing with a 4 mm FWHM Gaussian of 9 taps per axis
 * (CreateSmoothingFilters from the voxel sizes, :11055-11091); the sum of
 * the smoothed volume in the reference's order -- over x for every (y, z)
 * (CalculateColumnSums, kernelMisc.cpp:193-212), over y for every z
 * (CalculateRowSums, :214-231), over z on the host (CalculateSum,
 * broccoli_lib.cpp:10846-10886); threshold 0.9 x sum / (W H D); mask 1
 * where the smoothed value is above it and 0.001 elsewhere
 * (ThresholdVolume, kernelMisc.cpp:305-327). */
void FN(orc_segment_epi)(const REAL* vol, int W, int H, int D, double vx, double vy, double vz,
                         REAL* mask) {
  const long V = (long)W * H * D;
  REAL fx[9], fy[9], fz[9];
  FN(orc_smoothing_filter_fwhm)(9, 4.0, vx, vy, vz, fx, fy, fz);
  REAL* sm = (REAL*)malloc(sizeof(REAL) * V);
  FN(orc_smooth3d)(vol, NULL, NULL, W, H, D, fx, fy, fz, sm);
  REAL sum = RZERO;
  for (int z = 0; z < D; z++) {
    REAL zs = RZERO;
    for (int y = 0; y < H; y++) {
      REAL ys = RZERO;
      for (int x = 0; x < W; x++) ys += sm[x + (long)y * W + (long)z * W * H];
      zs += ys;
    }
    sum += zs;
  }
  const REAL thr = (REAL)0.9f * sum / ((REAL)W * (REAL)H * (REAL)D);
  for (long i = 0; i < V; i++) mask[i] = sm[i] > thr ? RONE : (REAL)0.001f;
  free(sm);
}

#undef RSQRT
#undef RATAN2
#undef RCOS
#undef RFLOOR
#undef RHALF
#undef RONE
#undef RZERO
#undef FN
