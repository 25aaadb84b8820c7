// ref_shim.cpp -- runs the reference's own OpenCL C kernels on the CPU.
// TEST INFRASTRUCTURE ONLY.  Built by `make ref` into oracle/_ref/ from the
// kernel sources where they lie in the BROCCOLI tree (the Makefile turns the
// OpenCL vector literals `(float2)(a,b)` into make_float2(a,b) in _ref/; the
// sources are never copied into this repository).  The host loops below
// restate BROCCOLI_LIB's drivers (code/BROCCOLI_LIB/broccoli_lib.cpp, cited
// per function) and call the vendored Eigen exactly where the reference does.
// Its outputs cross-check the C restatement in orc_impl.h and seed the golden
// fixtures under tests/golden/.
#include <Eigen/Dense>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "clshim.hpp"

namespace clk {
#include "kernelConvolution_cl.cpp"
}
namespace clr {
#include "kernelRegistration_cl.cpp"
}
namespace clm {
static inline void atomic_max(volatile int* p, int v) {
  if (v > *p) *p = v;
}
#include "kernelMisc_cl.cpp"
}

namespace {

// Runs `body` once per work-item of an NDRange (global g, local l); groups
// along the slowest non-trivial dimension are spread over OpenMP threads.
template <class F>
void ndrange(int g0, int g1, int g2, int l0, int l1, int l2, F body, bool parallel = true) {
  const int n2 = g2 / l2;
#pragma omp parallel for schedule(static) if (parallel)
  for (int b2 = 0; b2 < n2; b2++)
    for (int b1 = 0; b1 < g1 / l1; b1++)
      for (int b0 = 0; b0 < g0 / l0; b0++)
        for (int i2 = 0; i2 < l2; i2++)
          for (int i1 = 0; i1 < l1; i1++)
            for (int i0 = 0; i0 < l0; i0++) {
              g_ndr.lid[0] = i0; g_ndr.lid[1] = i1; g_ndr.lid[2] = i2;
              g_ndr.grp[0] = b0; g_ndr.grp[1] = b1; g_ndr.grp[2] = b2;
              g_ndr.gid[0] = b0 * l0 + i0; g_ndr.gid[1] = b1 * l1 + i1; g_ndr.gid[2] = b2 * l2 + i2;
              g_ndr.lsz[0] = l0; g_ndr.lsz[1] = l1; g_ndr.lsz[2] = l2;
              body();
            }
}

int roundup(int n, int m) { return (n + m - 1) / m * m; }

const int NPARAM = 12;
const int NNZ = 30;

}  // namespace

extern "C" {

// NonseparableConvolution3D, broccoli_lib.cpp:4974-5027, with the
// GlobalMemory kernel (kernelConvolution.cpp:2802-2867).  filters: 3 x
// {re[343], im[343]}; out: 3 interleaved complex volumes.
void ref_filter3d(const float* vol, int W, int H, int D, const float* filters, float* out) {
  const long V = (long)W * H * D;
  std::memset(out, 0, sizeof(float) * 6 * V);
  float2* q1 = reinterpret_cast<float2*>(out);
  float2* q2 = q1 + V;
  float2* q3 = q2 + V;
  int z_offset = -3;
  for (int zz = 6; zz >= 0; zz--) {
    const float* f1r = filters + 0 * 686 + zz * 49;
    const float* f1i = filters + 0 * 686 + 343 + zz * 49;
    const float* f2r = filters + 1 * 686 + zz * 49;
    const float* f2i = filters + 1 * 686 + 343 + zz * 49;
    const float* f3r = filters + 2 * 686 + zz * 49;
    const float* f3i = filters + 2 * 686 + 343 + zz * 49;
    ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1, [&] {
      clk::Nonseparable3DConvolutionComplexThreeQuadratureFiltersGlobalMemory(
          q1, q2, q3, vol, f1r, f1i, f2r, f2i, f3r, f3i, z_offset, W, H, D);
    });
    z_offset++;
  }
}

// The normal-equation part of one AlignTwoVolumesLinear iteration,
// broccoli_lib.cpp:5315-5392: phase differences / certainties / gradients
// and the 2D -> 1D -> final reductions per axis, then the mirroring.
void ref_normal_equations(const float* q1, const float* q2, int W, int H, int D, float* A144,
                          float* h12) {
  const long V = (long)W * H * D;
  std::vector<float> pd(V, 0.f), cert(V, 0.f), grad(V, 0.f);
  std::vector<float> A2((long)H * D * NNZ, 0.f), h2((long)H * D * NPARAM, 0.f);
  std::vector<float> A1((long)D * NNZ, 0.f), h1((long)D * NPARAM, 0.f);
  const float2* Q1 = reinterpret_cast<const float2*>(q1);
  const float2* Q2 = reinterpret_cast<const float2*>(q2);
  const int gx = roundup(W, 16), gy = roundup(H, 16);
  for (int axis = 0; axis < 3; axis++) {
    const float2* a = Q1 + axis * V;
    const float2* c = Q2 + axis * V;
    ndrange(gx, gy, D, 16, 16, 1, [&] {
      clr::CalculatePhaseDifferencesAndCertainties(pd.data(), cert.data(), a, c, W, H, D);
    });
    ndrange(gx, gy, D, 16, 16, 1, [&] {
      if (axis == 0) clr::CalculatePhaseGradientsX(grad.data(), a, c, W, H, D);
      if (axis == 1) clr::CalculatePhaseGradientsY(grad.data(), a, c, W, H, D);
      if (axis == 2) clr::CalculatePhaseGradientsZ(grad.data(), a, c, W, H, D);
    });
    ndrange(H, D, 1, H, 1, 1, [&] {
      if (axis == 0)
        clr::CalculateAMatrixAndHVector2DValuesX(A2.data(), h2.data(), pd.data(), grad.data(), cert.data(), W, H, D, 7);
      if (axis == 1)
        clr::CalculateAMatrixAndHVector2DValuesY(A2.data(), h2.data(), pd.data(), grad.data(), cert.data(), W, H, D, 7);
      if (axis == 2)
        clr::CalculateAMatrixAndHVector2DValuesZ(A2.data(), h2.data(), pd.data(), grad.data(), cert.data(), W, H, D, 7);
    }, false);
  }
  ndrange(D, NNZ, 1, D, 1, 1, [&] { clr::CalculateAMatrix1DValues(A1.data(), A2.data(), W, H, D, 7); }, false);
  ndrange(D, NPARAM, 1, D, 1, 1, [&] { clr::CalculateHVector1DValues(h1.data(), h2.data(), W, H, D, 7); }, false);
  std::memset(A144, 0, sizeof(float) * 144);
  ndrange(NNZ, 1, 1, NNZ, 1, 1, [&] { clr::CalculateAMatrix(A144, A1.data(), W, H, D, 7); }, false);
  ndrange(NPARAM, 1, 1, NPARAM, 1, 1, [&] { clr::CalculateHVector(h12, h1.data(), W, H, D, 7); }, false);
  for (int j = 0; j < NPARAM; j++)
    for (int i = 0; i < NPARAM; i++) A144[j + i * NPARAM] = A144[i + j * NPARAM];
}

// SolveEquationSystem, broccoli_lib.cpp:17157-17186.
void ref_solve(const float* A, const float* h, int N, float* p) {
  Eigen::MatrixXd Am(N, N);
  Eigen::VectorXd hv(N);
  for (int i = 0; i < N; i++) {
    hv(i) = (double)h[i];
    for (int j = 0; j < N; j++) Am(i, j) = (double)A[i + j * N];
  }
  Eigen::VectorXd x = Am.fullPivHouseholderQr().solve(hv);
  for (int i = 0; i < N; i++) p[i] = (float)x(i);
}

// RemoveTransformationScaling, broccoli_lib.cpp:6153-6194.
void ref_remove_scaling(float* p) {
  Eigen::MatrixXd T(3, 3);
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) T(r, c) = (double)p[3 + r * 3 + c];
  for (int d = 0; d < 3; d++) T(d, d) += 1.0;
  Eigen::JacobiSVD<Eigen::MatrixXd> svd(T, Eigen::ComputeThinU | Eigen::ComputeThinV);
  Eigen::MatrixXd R = svd.matrixU() * svd.matrixV().transpose();
  for (int d = 0; d < 3; d++) R(d, d) -= 1.0;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) p[3 + r * 3 + c] = (float)R(r, c);
}

static Eigen::MatrixXd to_affine(const float* p, float tscale) {
  Eigen::MatrixXd M(4, 4);
  M(0, 0) = (double)(p[3] + 1.0f); M(0, 1) = (double)p[4]; M(0, 2) = (double)p[5];
  M(1, 0) = (double)p[6]; M(1, 1) = (double)(p[7] + 1.0f); M(1, 2) = (double)p[8];
  M(2, 0) = (double)p[9]; M(2, 1) = (double)p[10]; M(2, 2) = (double)(p[11] + 1.0f);
  if (tscale == 1.0f) {
    M(0, 3) = (double)p[0]; M(1, 3) = (double)p[1]; M(2, 3) = (double)p[2];
  } else {
    M(0, 3) = (double)(p[0] * tscale); M(1, 3) = (double)(p[1] * tscale); M(2, 3) = (double)(p[2] * tscale);
  }
  M(3, 0) = 0.0; M(3, 1) = 0.0; M(3, 2) = 0.0; M(3, 3) = 1.0;
  return M;
}

static void from_affine(const Eigen::MatrixXd& T, float* p) {
  p[0] = (float)T(0, 3); p[1] = (float)T(1, 3); p[2] = (float)T(2, 3);
  p[3] = (float)(T(0, 0) - 1.0); p[4] = (float)T(0, 1); p[5] = (float)T(0, 2);
  p[6] = (float)T(1, 0); p[7] = (float)(T(1, 1) - 1.0); p[8] = (float)T(1, 2);
  p[9] = (float)T(2, 0); p[10] = (float)T(2, 1); p[11] = (float)(T(2, 2) - 1.0);
}

// AddAffineRegistrationParameters, broccoli_lib.cpp:7252-7340.
void ref_add_affine(float* old12, const float* new12) {
  Eigen::MatrixXd T = to_affine(new12, 1.0f) * to_affine(old12, 1.0f);
  from_affine(T, old12);
}

// InvertAffineRegistrationParameters, broccoli_lib.cpp:7186-7250 (Eigen's
// 4x4 inverse in double).
void ref_invert_affine(const float* p12, float* inv12) {
  Eigen::MatrixXd M = to_affine(p12, 1.0f);
  Eigen::MatrixXd I = M.inverse();
  from_affine(I, inv12);
}

// The DEBUG outputs of AlignTwoVolumesLinear (broccoli_lib.cpp:5315-5354)
// for one filter pair: CalculatePhaseDifferencesAndCertainties and
// CalculatePhaseGradientsX/Y/Z (kernelRegistration.cpp:173-382) into
// zero-filled outputs (the gradient kernels leave the first and last sample
// along the axis unwritten).
void ref_phase_volumes(const float* q1, const float* q2, int W, int H, int D, int axis, float* pd,
                       float* cert, float* grad) {
  const long V = (long)W * H * D;
  std::memset(pd, 0, sizeof(float) * V);
  std::memset(cert, 0, sizeof(float) * V);
  std::memset(grad, 0, sizeof(float) * V);
  const float2* a = reinterpret_cast<const float2*>(q1);
  const float2* c = reinterpret_cast<const float2*>(q2);
  const int gx = roundup(W, 16), gy = roundup(H, 16);
  ndrange(gx, gy, D, 16, 16, 1, [&] { clr::CalculatePhaseDifferencesAndCertainties(pd, cert, a, c, W, H, D); });
  ndrange(gx, gy, D, 16, 16, 1, [&] {
    if (axis == 0) clr::CalculatePhaseGradientsX(grad, a, c, W, H, D);
    if (axis == 1) clr::CalculatePhaseGradientsY(grad, a, c, W, H, D);
    if (axis == 2) clr::CalculatePhaseGradientsZ(grad, a, c, W, H, D);
  });
}

// AddAffineRegistrationParametersNextScale, broccoli_lib.cpp:7344-7431.
void ref_add_affine_next_scale(float* old12, const float* new12) {
  Eigen::MatrixXd T = to_affine(new12, 2.0f) * to_affine(old12, 2.0f);
  from_affine(T, old12);
}

// CalculateRotationAnglesFromRotationMatrix, broccoli_lib.cpp:6199-6244.
void ref_rotation_angles(const float* p, float* rot) {
  const double PI_ = 3.14159265358979323846;
  double m[9];
  for (int i = 3; i < 12; i++) m[i - 3] = (double)p[i];
  m[0] += 1.0; m[4] += 1.0; m[8] += 1.0;
  const double a1 = -atan2(m[5], m[8]) * 180.0 / PI_;
  const double c2 = sqrt(m[0] * m[0] + m[1] * m[1]);
  const double a2 = -atan2(-m[2], c2) * 180.0 / PI_;
  const double s1 = sin(a1 * PI_ / 180.0), c1 = cos(a1 * PI_ / 180.0);
  const double a3 = -atan2(s1 * m[6] - c1 * m[3], c1 * m[4] - s1 * m[7]) * 180.0 / PI_;
  rot[0] = (float)a1; rot[1] = (float)a2; rot[2] = (float)a3;
}

// InterpolateVolumeLinearLinear (kernelRegistration.cpp:1066-1101) as driven
// at broccoli_lib.cpp:5424-5427.
void ref_warp_affine(const float* src, int W, int H, int D, const float* p12, float* out) {
  const image3d_t im{src, W, H, D};
  ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1,
          [&] { clr::InterpolateVolumeLinearLinear(out, im, p12, W, H, D, 0); });
}

// InterpolateVolumeLinearNonLinear, kernelRegistration.cpp:1111-1140.
void ref_warp_field(const float* src, int W, int H, int D, const float* dx, const float* dy,
                    const float* dz, float* out) {
  const image3d_t im{src, W, H, D};
  ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1,
          [&] { clr::InterpolateVolumeLinearNonLinear(out, im, dx, dy, dz, W, H, D, 0); });
}

// ChangeVolumeSize with LINEAR interpolation, broccoli_lib.cpp:6247-6388.
void ref_rescale_linear(const float* src, int W, int H, int D, int W2, int H2, int D2, float* out) {
  const image3d_t im{src, W, H, D};
  const float vx = (float)(W - 1) / (float)(W2 - 1);
  const float vy = (float)(H - 1) / (float)(H2 - 1);
  const float vz = (float)(D - 1) / (float)(D2 - 1);
  ndrange(roundup(W2, 16), roundup(H2, 16), D2, 16, 16, 1,
          [&] { clr::RescaleVolumeLinear(out, im, vx, vy, vz, W2, H2, D2); });
}

// TransformVolumesLinear, broccoli_lib.cpp:8267-8359: the volumes one after
// another through InterpolateVolumeNearestLinear (interp 0) or
// InterpolateVolumeLinearLinear (1), kernelRegistration.cpp:995-1101.
void ref_transform_linear(const float* src, int W, int H, int D, int T, const float* p12, int interp,
                          float* out) {
  const long V = (long)W * H * D;
  for (int t = 0; t < T; t++) {
    const image3d_t im{src + t * V, W, H, D};
    ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1, [&] {
      if (interp == 0)
        clr::InterpolateVolumeNearestLinear(out, im, p12, W, H, D, t);
      else
        clr::InterpolateVolumeLinearLinear(out, im, p12, W, H, D, t);
    });
  }
}

// TransformVolumesNonLinear, broccoli_lib.cpp:8361-8451
// (InterpolateVolumeNearestNonLinear / LinearNonLinear).
void ref_transform_nonlinear(const float* src, int W, int H, int D, int T, const float* dx, const float* dy,
                             const float* dz, int interp, float* out) {
  const long V = (long)W * H * D;
  for (int t = 0; t < T; t++) {
    const image3d_t im{src + t * V, W, H, D};
    ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1, [&] {
      if (interp == 0)
        clr::InterpolateVolumeNearestNonLinear(out, im, dx, dy, dz, W, H, D, t);
      else
        clr::InterpolateVolumeLinearNonLinear(out, im, dx, dy, dz, W, H, D, t);
    });
  }
}

// AlignTwoVolumesLinear, broccoli_lib.cpp:5273-5437 (type 0 TRANSLATION,
// 1 RIGID, 2 AFFINE).  `aligned` is updated in place; `original` is the
// image that is re-sampled each iteration.
void ref_align_linear(const float* ref, float* aligned, const float* original, int W, int H, int D,
                      const float* filters, int niter, int type, float* p12, float* rot3) {
  const long V = (long)W * H * D;
  std::vector<float> q1(6 * V), q2(6 * V);
  float A[144], h[12], p[12];
  ref_filter3d(ref, W, H, D, filters, q1.data());
  for (int i = 0; i < 12; i++) p12[i] = 0.f;
  for (int it = 0; it < niter; it++) {
    ref_filter3d(aligned, W, H, D, filters, q2.data());
    ref_normal_equations(q1.data(), q2.data(), W, H, D, A, h);
    ref_solve(A, h, 12, p);
    if (type == 0) {
      p12[0] += p[0]; p12[1] += p[1]; p12[2] += p[2];
      for (int i = 3; i < 12; i++) p12[i] = 0.f;
    } else if (type == 1) {
      ref_remove_scaling(p);
      ref_add_affine(p12, p);
    } else {
      ref_add_affine(p12, p);
    }
    ref_warp_affine(original, W, H, D, p12, aligned);
  }
  if (type == 1 && rot3) ref_rotation_angles(p12, rot3);
}

// PerformMotionCorrectionWrapper, broccoli_lib.cpp:10658-10720 (reference =
// volume 0; the reference volume is refiltered for every volume, as there).
void ref_motion_correct(float* vols, int W, int H, int D, int T, const float* voxel_size,
                        const float* filters, int niter, float* motion6T) {
  const long V = (long)W * H * D;
  std::vector<float> ref(vols, vols + V), orig(V);
  for (int k = 0; k < 6; k++) motion6T[k * T] = 0.f;
  for (int t = 1; t < T; t++) {
    float p[12], rot[3];
    float* vt = vols + (long)t * V;
    std::memcpy(orig.data(), vt, sizeof(float) * V);
    ref_align_linear(ref.data(), vt, orig.data(), W, H, D, filters, niter, 1, p, rot);
    motion6T[t + 0 * T] = p[0] * voxel_size[0];
    motion6T[t + 1 * T] = p[1] * voxel_size[1];
    motion6T[t + 2 * T] = p[2] * voxel_size[2];
    motion6T[t + 3 * T] = rot[0];
    motion6T[t + 4 * T] = rot[1];
    motion6T[t + 5 * T] = rot[2];
  }
}

// PerformSmoothing (broccoli_lib.cpp:11274-11357): Rows (x certainty),
// Columns, Rods (/ smoothed certainty) with the GlobalMemory kernels
// (kernelConvolution.cpp:52-91, :531-569, :1201-1240).  cert and
// smoothed_cert may be NULL for all-ones.
void ref_smooth3d(const float* vol, const float* cert, const float* scert, int W, int H, int D,
                  const float* fx, const float* fy, const float* fz, float* out) {
  const long V = (long)W * H * D;
  std::vector<float> ones, rows(V), cols(V);
  if (!cert || !scert) ones.assign(V, 1.f);
  const float* c = cert ? cert : ones.data();
  const float* sc = scert ? scert : ones.data();
  const int gx = roundup(W, 16), gy = roundup(H, 16);
  ndrange(gx, gy, D, 16, 16, 1,
          [&] { clk::SeparableConvolutionRowsGlobalMemory(rows.data(), vol, c, fy, 0, W, H, D, 1); });
  ndrange(gx, gy, D, 16, 16, 1,
          [&] { clk::SeparableConvolutionColumnsGlobalMemory(cols.data(), rows.data(), fx, 0, W, H, D, 1); });
  ndrange(gx, gy, D, 16, 16, 1,
          [&] { clk::SeparableConvolutionRodsGlobalMemory(out, cols.data(), sc, fz, 0, W, H, D, 1); });
}

static void smooth_inplace(float* vol, int W, int H, int D, const float* f) {
  const long V = (long)W * H * D;
  std::vector<float> out(V);
  ref_smooth3d(vol, nullptr, nullptr, W, H, D, f, f, f, out.data());
  std::memcpy(vol, out.data(), sizeof(float) * V);
}

static void smoothing_filter(double sigma, float* f) {
  // CreateSmoothingFilters(..., double sigma), broccoli_lib.cpp:11093-11121
  const double s2 = 2.0 * sigma * sigma;
  float sum = 0.0f;
  for (int i = 0; i < 9; i++) {
    const double u = (double)(i - 4);
    f[i] = (float)exp(-pow(u, 2.0) / s2);
    sum += f[i];
  }
  for (int i = 0; i < 9; i++) f[i] /= sum;
}

// AlignTwoVolumesNonLinear, broccoli_lib.cpp:5748-6058, with the
// reference's kernels (kernelRegistration.cpp:806-988, kernelMisc.cpp
// CalculateColumnMaxs/RowMaxs, AddVolumes, MultiplyVolume) and the host max
// of CalculateMax (broccoli_lib.cpp:10889-10928).  field: 3 volumes.
void ref_align_nonlinear(const float* ref, float* aligned, const float* original, int W, int H,
                         int D, const float* filters6, const float* tensors, const float* dirs,
                         int niter, double tsigma, double esigma, double dsigma, float* field) {
  const long V = (long)W * H * D;
  std::vector<float> q1(12 * V), q2(12 * V), t(6 * V), a(6 * V), h(3 * V), d(3 * V), tmp(V);
  std::vector<float> colmax((long)H * D), maxs(D);
  ref_filter3d(ref, W, H, D, filters6, q1.data());
  ref_filter3d(ref, W, H, D, filters6 + 3 * 686, q1.data() + 6 * V);
  std::memset(field, 0, sizeof(float) * 3 * V);
  float ft[9], fe[9], fd[9];
  smoothing_filter(tsigma, ft);
  smoothing_filter(esigma, fe);
  smoothing_filter(dsigma, fd);
  const int gx = roundup(W, 16), gy = roundup(H, 16);
  const float2* Q1 = reinterpret_cast<const float2*>(q1.data());
  const float2* Q2 = reinterpret_cast<const float2*>(q2.data());
  float *t11 = t.data(), *t12 = t11 + V, *t13 = t12 + V, *t22 = t13 + V, *t23 = t22 + V, *t33 = t23 + V;
  float *a11 = a.data(), *a12 = a11 + V, *a13 = a12 + V, *a22 = a13 + V, *a23 = a22 + V, *a33 = a23 + V;
  float *h1 = h.data(), *h2 = h1 + V, *h3 = h2 + V;
  float *dx = d.data(), *dy = dx + V, *dz = dy + V;
  const image3d_t im{original, W, H, D};
  for (int it = 0; it < niter; it++) {
    ref_filter3d(aligned, W, H, D, filters6, q2.data());
    ref_filter3d(aligned, W, H, D, filters6 + 3 * 686, q2.data() + 6 * V);
    std::fill(t.begin(), t.end(), 0.f);
    std::fill(a.begin(), a.end(), 0.f);
    std::fill(h.begin(), h.end(), 0.f);
    for (int k = 0; k < 6; k++) {
      const float* m = tensors + 6 * k;
      ndrange(gx, gy, D, 16, 16, 1, [&] {
        clr::CalculateTensorComponents(t11, t12, t13, t22, t23, t33, Q1 + k * V, Q2 + k * V, m[0], m[1],
                                       m[2], m[3], m[4], m[5], W, H, D);
      });
    }
    ndrange(gx, gy, D, 16, 16, 1, [&] { clr::CalculateTensorNorms(a11, t11, t12, t13, t22, t23, t33, W, H, D); });
    for (int c = 0; c < 6; c++) smooth_inplace(t.data() + c * V, W, H, D, ft);
    ndrange(gx, gy, D, 16, 16, 1, [&] { clr::CalculateTensorNorms(a11, t11, t12, t13, t22, t23, t33, W, H, D); });
    ndrange(roundup(H, 16), roundup(D, 16), 1, 16, 16, 1,
            [&] { clm::CalculateColumnMaxs(colmax.data(), a11, W, H, D); }, false);
    ndrange(roundup(D, 16), 1, 1, 16, 1, 1, [&] { clm::CalculateRowMaxs(maxs.data(), colmax.data(), H, D); }, false);
    float mx = std::numeric_limits<float>::min();
    for (int z = 0; z < D; z++) mx = clm::mymax(mx, maxs[z]);
    const float f = 1.0f / mx;
    for (int c = 0; c < 6; c++) {
      float* tc = t.data() + c * V;
      ndrange(gx, gy, D, 16, 16, 1, [&] { clm::MultiplyVolume(tc, f, W, H, D); });
    }
    for (int k = 0; k < 6; k++) {
      ndrange(gx, gy, D, 16, 16, 1, [&] {
        clr::CalculateAMatricesAndHVectors(a11, a12, a13, a22, a23, a33, h1, h2, h3, Q1 + k * V, Q2 + k * V,
                                           t11, t12, t13, t22, t23, t33, dirs, dirs + 6, dirs + 12, W, H, D, k);
      });
    }
    for (int c = 0; c < 6; c++) smooth_inplace(a.data() + c * V, W, H, D, fe);
    for (int c = 0; c < 3; c++) smooth_inplace(h.data() + c * V, W, H, D, fe);
    ndrange(gx, gy, D, 16, 16, 1, [&] {
      clr::CalculateDisplacementUpdate(dx, dy, dz, a11, a12, a13, a22, a23, a33, h1, h2, h3, W, H, D);
    });
    for (int c = 0; c < 3; c++) {
      smooth_inplace(d.data() + c * V, W, H, D, fd);
      float* fc = field + c * V;
      const float* dc = d.data() + c * V;
      ndrange(gx, gy, D, 16, 16, 1, [&] { clm::AddVolumesOverwrite(fc, dc, W, H, D); });
    }
    ndrange(gx, gy, D, 16, 16, 1, [&] {
      clr::InterpolateVolumeLinearNonLinear(aligned, im, field, field + V, field + 2 * V, W, H, D, 0);
    });
  }
}

static int myround_(float a) { return (int)floorf(a + 0.5f); }

// ChangeVolumesResolutionAndSize, broccoli_lib.cpp:6950-7100: the
// reference's RescaleVolumeLinear then CopyVolumeToNew kernels.
void ref_change_resolution_and_size(const float* src, int W, int H, int D, float vx, float vy, float vz,
                                    float* out, int W2, int H2, int D2, float nvx, float nvy, float nvz,
                                    int mm_z_cut) {
  const int Wi = myround_((float)W * vx / nvx), Hi = myround_((float)H * vy / nvy),
            Di = myround_((float)D * vz / nvz);
  std::vector<float> interp((long)Wi * Hi * Di, 0.f);
  ref_rescale_linear(src, W, H, D, Wi, Hi, Di, interp.data());
  std::memset(out, 0, sizeof(float) * (long)W2 * H2 * D2);
  const int gx = W2 > Wi ? W2 : Wi, gy = H2 > Hi ? H2 : Hi, gz = D2 > Di ? D2 : Di;
  ndrange(roundup(gx, 16), roundup(gy, 16), gz, 16, 16, 1, [&] {
    clr::CopyVolumeToNew(out, interp.data(), W2, H2, D2, Wi, Hi, Di, Wi - W2, Hi - H2, Di - D2, mm_z_cut,
                         nvz, 0);
  });
}

// ChangeVolumesResolutionAndSize with INTERPOLATION_MODE 0 (RescaleVolumeNearest,
// kernelRegistration.cpp:1312-1338) or 1 (RescaleVolumeLinear) for T volumes,
// broccoli_lib.cpp:6950-7100.
void ref_change_resolution_and_size_interp(const float* src, int W, int H, int D, int T, float vx, float vy,
                                           float vz, float* out, int W2, int H2, int D2, float nvx, float nvy,
                                           float nvz, int mm_z_cut, int interp) {
  const int Wi = myround_((float)W * vx / nvx), Hi = myround_((float)H * vy / nvy),
            Di = myround_((float)D * vz / nvz);
  const float rx = (float)(W - 1) / (float)(Wi - 1), ry = (float)(H - 1) / (float)(Hi - 1),
              rz = (float)(D - 1) / (float)(Di - 1);
  const long V = (long)W * H * D, V2 = (long)W2 * H2 * D2;
  std::vector<float> interp_v((long)Wi * Hi * Di, 0.f);
  for (int t = 0; t < T; t++) {
    const image3d_t im{src + t * V, W, H, D};
    ndrange(roundup(Wi, 16), roundup(Hi, 16), Di, 16, 16, 1, [&] {
      if (interp == 0)
        clr::RescaleVolumeNearest(interp_v.data(), im, rx, ry, rz, Wi, Hi, Di);
      else
        clr::RescaleVolumeLinear(interp_v.data(), im, rx, ry, rz, Wi, Hi, Di);
    });
    float* o = out + t * V2;
    std::memset(o, 0, sizeof(float) * V2);
    const int gx = W2 > Wi ? W2 : Wi, gy = H2 > Hi ? H2 : Hi, gz = D2 > Di ? D2 : Di;
    ndrange(roundup(gx, 16), roundup(gy, 16), gz, 16, 16, 1, [&] {
      clr::CopyVolumeToNew(o, interp_v.data(), W2, H2, D2, Wi, Hi, Di, Wi - W2, Hi - H2, Di - D2, mm_z_cut,
                           nvz, 0);
    });
  }
}

// CalculateCenterOfMass, broccoli_lib.cpp:6763-6800 (host loop).
static void com_(const float* v, int W, int H, int D, float* c) {
  float tm = 0.f, rx = 0.f, ry = 0.f, rz = 0.f;
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const float m = v[x + (long)y * W + (long)z * W * H];
        rx += m * (float)x;
        ry += m * (float)y;
        rz += m * (float)z;
        tm += m;
      }
  c[0] = rx / tm;
  c[1] = ry / tm;
  c[2] = rz / tm;
}

// MatchVolumeMasses, broccoli_lib.cpp:6876-6948, with
// TransformVolumesLinear (InterpolateVolumeLinearLinear).
void ref_match_volume_masses(float* v1, const float* v2, int W, int H, int D, float* p12) {
  float c1[3], c2[3];
  com_(v1, W, H, D, c1);
  com_(v2, W, H, D, c2);
  for (int i = 0; i < 12; i++) p12[i] = 0.f;
  p12[0] = -(float)myround_(c2[0] - c1[0]);
  p12[1] = -(float)myround_(c2[1] - c1[1]);
  p12[2] = -(float)myround_(c2[2] - c1[2]);
  std::vector<float> tmp(v1, v1 + (long)W * H * D);
  ref_warp_affine(tmp.data(), W, H, D, p12, v1);
}

// CenterVolumesWrapper, broccoli_lib.cpp:8225-8245, with CenterVolumeMass
// (:6839-6874): translation from the first volume's centre of mass, then
// TransformVolumesLinear of all T volumes.
void ref_center_volumes(const float* src, int W, int H, int D, int T, int interp, float* out, float* p12) {
  float c[3];
  com_(src, W, H, D, c);
  for (int i = 0; i < 12; i++) p12[i] = 0.f;
  p12[0] = -(float)myround_((float)W / 2.0f - c[0]);
  p12[1] = -(float)myround_((float)H / 2.0f - c[1]);
  p12[2] = -(float)myround_((float)D / 2.0f - c[2]);
  ref_transform_linear(src, W, H, D, T, p12, interp, out);
}

// CreateCombinedDisplacementField, broccoli_lib.cpp:8115-8150, with
// AddLinearAndNonLinearDisplacement (kernelRegistration.cpp:1142-1178).
void ref_add_linear_nonlinear(float* field, int W, int H, int D, const float* p12) {
  const long V = (long)W * H * D;
  ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1, [&] {
    clr::AddLinearAndNonLinearDisplacement(field, field + V, field + 2 * V, p12, W, H, D);
  });
}

// AlignTwoVolumesLinearSeveralScales, broccoli_lib.cpp:6391-6513, around
// the reference kernels (ChangeVolumeSize = RescaleVolumeLinear,
// InterpolateVolumeLinearLinear).  `aligned` in: moving volume, out: the
// moving volume warped by the total parameters (DO_OVERWRITE).
void ref_align_linear_scales(const float* ref, float* aligned, int W, int H, int D, int coarsest,
                             const float* filters, int niter, int type, float* p12, float* rot3) {
  const long V = (long)W * H * D;
  std::vector<float> orig(aligned, aligned + V), r_s(V), o_s(V), a_s(V), resc(V);
  float tmp[12], rt[3] = {0.f, 0.f, 0.f};
  for (int i = 0; i < 12; i++) p12[i] = 0.f;
  rot3[0] = rot3[1] = rot3[2] = 0.f;
  int cw = myround_((float)W / (float)coarsest), ch = myround_((float)H / (float)coarsest),
      cd = myround_((float)D / (float)coarsest);
  ref_rescale_linear(orig.data(), W, H, D, cw, ch, cd, o_s.data());
  ref_rescale_linear(ref, W, H, D, cw, ch, cd, r_s.data());
  for (int scale = coarsest; scale >= 1; scale /= 2) {
    const long vs = (long)cw * ch * cd;
    std::memcpy(a_s.data(), o_s.data(), sizeof(float) * vs);
    const int it = scale == 1 ? (int)ceilf((float)niter / 5.0f) : niter;
    ref_align_linear(r_s.data(), a_s.data(), o_s.data(), cw, ch, cd, filters, it, type, tmp, rt);
    if (type != 1) rt[0] = rt[1] = rt[2] = 0.f;
    if (scale != 1) {
      rot3[0] += rt[0]; rot3[1] += rt[1]; rot3[2] += rt[2];
      ref_add_affine_next_scale(p12, tmp);
      cw = myround_((float)W / ((float)scale / 2.0f));
      ch = myround_((float)H / ((float)scale / 2.0f));
      cd = myround_((float)D / ((float)scale / 2.0f));
      ref_rescale_linear(orig.data(), W, H, D, cw, ch, cd, resc.data());
      ref_rescale_linear(ref, W, H, D, cw, ch, cd, r_s.data());
      ref_warp_affine(resc.data(), cw, ch, cd, p12, o_s.data());
    } else {
      ref_add_affine(p12, tmp);
      rot3[0] += rt[0]; rot3[1] += rt[1]; rot3[2] += rt[2];
      ref_warp_affine(orig.data(), W, H, D, p12, aligned);
    }
  }
}

// AlignTwoVolumesNonLinearSeveralScales, broccoli_lib.cpp:6516-6665.
void ref_align_nonlinear_scales(const float* ref, float* aligned, int W, int H, int D, int coarsest,
                                const float* filters6, const float* tensors, const float* dirs,
                                int niter, double tsigma, double esigma, double dsigma, float* field) {
  const long V = (long)W * H * D;
  std::vector<float> orig(aligned, aligned + V), r_s(V), o_s(V), a_s(V), resc(V);
  std::vector<float> tot(3 * V, 0.f), upd(3 * V), tmp(3 * V);
  int cw = myround_((float)W / (float)coarsest), ch = myround_((float)H / (float)coarsest),
      cd = myround_((float)D / (float)coarsest);
  ref_rescale_linear(orig.data(), W, H, D, cw, ch, cd, o_s.data());
  ref_rescale_linear(ref, W, H, D, cw, ch, cd, r_s.data());
  for (int scale = coarsest; scale >= 1; scale /= 2) {
    const long vs = (long)cw * ch * cd;
    std::memcpy(a_s.data(), o_s.data(), sizeof(float) * vs);
    const int it = scale == 1 ? (int)ceilf((float)niter / 2.0f) : niter;
    ref_align_nonlinear(r_s.data(), a_s.data(), o_s.data(), cw, ch, cd, filters6, tensors, dirs, it,
                        tsigma, esigma, dsigma, upd.data());
    for (int c = 0; c < 3; c++) {
      float* t = tot.data() + c * vs;
      const float* u = upd.data() + c * vs;
      ndrange(roundup(cw, 16), roundup(ch, 16), cd, 16, 16, 1, [&] { clm::AddVolumesOverwrite(t, u, cw, ch, cd); });
    }
    if (scale != 1) {
      const int pw = cw, ph = ch, pdp = cd;
      cw = myround_((float)W / ((float)scale / 2.0f));
      ch = myround_((float)H / ((float)scale / 2.0f));
      cd = myround_((float)D / ((float)scale / 2.0f));
      const long nv = (long)cw * ch * cd;
      for (int c = 0; c < 3; c++) {
        ref_rescale_linear(tot.data() + c * (long)pw * ph * pdp, pw, ph, pdp, cw, ch, cd, tmp.data() + c * nv);
        float* t = tmp.data() + c * nv;
        ndrange(roundup(cw, 16), roundup(ch, 16), cd, 16, 16, 1, [&] { clm::MultiplyVolume(t, 2.0f, cw, ch, cd); });
      }
      std::memcpy(tot.data(), tmp.data(), sizeof(float) * 3 * nv);
      ref_rescale_linear(orig.data(), W, H, D, cw, ch, cd, resc.data());
      ref_rescale_linear(ref, W, H, D, cw, ch, cd, r_s.data());
      ref_warp_field(resc.data(), cw, ch, cd, tot.data(), tot.data() + nv, tot.data() + 2 * nv, o_s.data());
    } else {
      std::memcpy(field, tot.data(), sizeof(float) * 3 * V);
      ref_warp_field(orig.data(), W, H, D, field, field + V, field + 2 * V, aligned);
    }
  }
}

// PerformRegistrationTwoVolumesWrapper, broccoli_lib.cpp:7973-8112 (one
// volume, no pre-centring, no skull strip).
void ref_register_two_volumes(const float* in, int W, int H, int D, const float* vin, const float* tpl,
                              int W2, int H2, int D2, const float* vtpl, int mm_z_cut, int coarsest,
                              int lin_iter, int nl_iter, const float* filters3, const float* filters6,
                              const float* tensors, const float* dirs, double tsigma, double esigma,
                              double dsigma, float* p12, float* interpolated, float* aligned_linear,
                              float* aligned_nonlinear, float* field) {
  const long V2 = (long)W2 * H2 * D2;
  std::vector<float> work(V2);
  float match[12], rot[3];
  ref_change_resolution_and_size(in, W, H, D, vin[0], vin[1], vin[2], work.data(), W2, H2, D2, vtpl[0],
                                 vtpl[1], vtpl[2], mm_z_cut);
  ref_match_volume_masses(work.data(), tpl, W2, H2, D2, match);
  std::memcpy(interpolated, work.data(), sizeof(float) * V2);
  ref_align_linear_scales(tpl, work.data(), W2, H2, D2, coarsest, filters3, lin_iter, 2, p12, rot);
  std::memcpy(aligned_linear, work.data(), sizeof(float) * V2);
  ref_add_affine(p12, match);
  ref_align_nonlinear_scales(tpl, work.data(), W2, H2, D2, coarsest, filters6, tensors, dirs, nl_iter,
                             tsigma, esigma, dsigma, field);
  ref_add_linear_nonlinear(field, W2, H2, D2, p12);
  ref_change_resolution_and_size(in, W, H, D, vin[0], vin[1], vin[2], work.data(), W2, H2, D2, vtpl[0],
                                 vtpl[1], vtpl[2], mm_z_cut);
  ref_warp_field(work.data(), W2, H2, D2, field, field + V2, field + 2 * V2, aligned_nonlinear);
}

// CalculateTensorMagnitude, broccoli_lib.cpp:5658-5746, with the
// reference's CalculateTensorComponents and CalculateTensorNorms kernels.
void ref_tensor_magnitude(const float* vol, int W, int H, int D, const float* filters6, const float* tensors,
                          float* out) {
  const long V = (long)W * H * D;
  std::vector<float> q(12 * V), t(6 * V, 0.f);
  ref_filter3d(vol, W, H, D, filters6, q.data());
  ref_filter3d(vol, W, H, D, filters6 + 3 * 686, q.data() + 6 * V);
  const float2* Q = reinterpret_cast<const float2*>(q.data());
  float *t11 = t.data(), *t12 = t11 + V, *t13 = t12 + V, *t22 = t13 + V, *t23 = t22 + V, *t33 = t23 + V;
  const int gx = roundup(W, 16), gy = roundup(H, 16);
  for (int k = 0; k < 6; k++) {
    const float* m = tensors + 6 * k;
    ndrange(gx, gy, D, 16, 16, 1, [&] {
      clr::CalculateTensorComponents(t11, t12, t13, t22, t23, t33, Q + k * V, Q + k * V, m[0], m[1], m[2], m[3],
                                     m[4], m[5], W, H, D);
    });
  }
  ndrange(gx, gy, D, 16, 16, 1, [&] { clr::CalculateTensorNorms(out, t11, t12, t13, t22, t23, t33, W, H, D); });
}

// SegmentEPIData, broccoli_lib.cpp:11008-11030: 4 mm FWHM smoothing
// (CreateSmoothingFilters, :11055-11091, restated), CalculateSum
// (:10846-10886) on the reference's CalculateColumnSums / CalculateRowSums
// kernels, and its ThresholdVolume kernel at 0.9 x the mean.
void ref_segment_epi(const float* vol, int W, int H, int D, double vx, double vy, double vz, float* mask) {
  const long V = (long)W * H * D;
  float f[3][9];
  const double vs[3] = {vx, vy, vz};
  for (int a = 0; a < 3; a++) {
    const double s = 4.0 / 2.354 / vs[a];
    const double s2 = 2.0 * s * s;
    float sum = 0.0f;
    for (int i = 0; i < 9; i++) {
      const double u = (double)(i - 4);
      f[a][i] = (float)exp(-pow(u, 2.0) / s2);
      sum += f[a][i];
    }
    for (int i = 0; i < 9; i++) f[a][i] /= sum;
  }
  std::vector<float> sm(V), cols((long)H * D), rows(D);
  ref_smooth3d(vol, nullptr, nullptr, W, H, D, f[0], f[1], f[2], sm.data());
  ndrange(roundup(H, 16), roundup(D, 16), 1, 16, 16, 1,
          [&] { clm::CalculateColumnSums(cols.data(), sm.data(), W, H, D); }, false);
  ndrange(roundup(D, 16), 1, 1, 16, 1, 1, [&] { clm::CalculateRowSums(rows.data(), cols.data(), H, D); }, false);
  float sum = 0.0f;
  for (int z = 0; z < D; z++) sum += rows[z];
  const float thr = 0.9f * sum / ((float)W * H * D);
  ndrange(roundup(W, 16), roundup(H, 16), D, 16, 16, 1,
          [&] { clm::ThresholdVolume(mask, sm.data(), thr, W, H, D); });
}

}  // extern "C"
