// drift_adjoint.cu -- discrete adjoint of the taped DOP853 integration.
//
// The forward kernel (drift_kernels.cuh with a tape) records for every
// accepted step of every particle (t_old, h, y_old).  With the step sizes
// held fixed, the trajectory is a composition of explicit maps:
//   stages   z_i = y + h sum_j a_ij k_j,  k_i = f(z_i)       (i = 2..12)
//   solution y_new = y + h sum_j b_j k_j,  k_13 = f(y_new)   (FSAL, the next k_1)
//   dense    z_i, k_i for i = 14..16, rcont1..8 and the interpolant
//            y(t) = r1 + s(r2 + s1(r3 + s(r4 + s1(r5 + s(r6 + s1(r7 + s r8))))))
// (src/integrators/galpy/dop853.rs:425-763, Hairer's stage numbering; the
// forward code reuses the names k2, k3, k4, k10 for stages 11-16).  This
// kernel runs each particle's steps in reverse, recomputes one step's stages
// from its tape row and propagates the cotangents through the maps above,
// with hand-written vector-Jacobian products of f = (v, a(x)):
//   lambda_x += J_a(x)^T lambda_v,  lambda_v += lambda_x,
// and the force's parameter derivatives (drift_jacobians.cuh).  The result
// is the exact derivative of the computed trajectory for the recorded step
// sequence (the step-size controller is not differentiated).
//
// Compiled with multiply-add contraction (a gradient has no bit-parity
// requirement); one thread per particle, grid-stride.
#define DRIFT_EXACT_ARITH 0

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>

#include "drift_b200.h"
#include "drift_common.cuh"
#include "drift_dop853.cuh"
#include "drift_jacobians.cuh"
#include "drift_launch_args.cuh"
#include "drift_trace.h"

int drift_internal_fail(int code, const char *msg);

namespace drift {
namespace adjoint {

using namespace dop853c;

// Stage-input coefficients a_ij (Hairer numbering; 13 is the FSAL stage).
__host__ __device__ constexpr double acoef(int i, int j)
{
    switch (i * 100 + j) {
    case 201: return A21;
    case 301: return A31;
    case 302: return A32;
    case 401: return A41;
    case 403: return A43;
    case 501: return A51;
    case 503: return A53;
    case 504: return A54;
    case 601: return A61;
    case 604: return A64;
    case 605: return A65;
    case 701: return A71;
    case 704: return A74;
    case 705: return A75;
    case 706: return A76;
    case 801: return A81;
    case 804: return A84;
    case 805: return A85;
    case 806: return A86;
    case 807: return A87;
    case 901: return A91;
    case 904: return A94;
    case 905: return A95;
    case 906: return A96;
    case 907: return A97;
    case 908: return A98;
    case 1001: return A101;
    case 1004: return A104;
    case 1005: return A105;
    case 1006: return A106;
    case 1007: return A107;
    case 1008: return A108;
    case 1009: return A109;
    case 1101: return A111;
    case 1104: return A114;
    case 1105: return A115;
    case 1106: return A116;
    case 1107: return A117;
    case 1108: return A118;
    case 1109: return A119;
    case 1110: return A1110;
    case 1201: return A121;
    case 1204: return A124;
    case 1205: return A125;
    case 1206: return A126;
    case 1207: return A127;
    case 1208: return A128;
    case 1209: return A129;
    case 1210: return A1210;
    case 1211: return A1211;
    case 1401: return A141;
    case 1407: return A147;
    case 1408: return A148;
    case 1409: return A149;
    case 1410: return A1410;
    case 1411: return A1411;
    case 1412: return A1412;
    case 1413: return A1413;
    case 1501: return A151;
    case 1506: return A156;
    case 1507: return A157;
    case 1508: return A158;
    case 1511: return A1511;
    case 1512: return A1512;
    case 1513: return A1513;
    case 1514: return A1514;
    case 1601: return A161;
    case 1606: return A166;
    case 1607: return A167;
    case 1608: return A168;
    case 1609: return A169;
    case 1613: return A1613;
    case 1614: return A1614;
    case 1615: return A1615;
    default: return 0.0;
    }
}

// Solution weights b_j.
__host__ __device__ constexpr double bcoef(int j)
{
    switch (j) {
    case 1: return B1;
    case 6: return B6;
    case 7: return B7;
    case 8: return B8;
    case 9: return B9;
    case 10: return B10;
    case 11: return B11;
    case 12: return B12;
    default: return 0.0;
    }
}

// rcont5..8 = h sum_j d_mj k_j (m = 5..8).
__host__ __device__ constexpr double dcoef(int m, int j)
{
    switch (m * 100 + j) {
    case 501: return D41;
    case 506: return D46;
    case 507: return D47;
    case 508: return D48;
    case 509: return D49;
    case 510: return D410;
    case 511: return D411;
    case 512: return D412;
    case 513: return D413;
    case 514: return D414;
    case 515: return D415;
    case 516: return D416;
    case 601: return D51;
    case 606: return D56;
    case 607: return D57;
    case 608: return D58;
    case 609: return D59;
    case 610: return D510;
    case 611: return D511;
    case 612: return D512;
    case 613: return D513;
    case 614: return D514;
    case 615: return D515;
    case 616: return D516;
    case 701: return D61;
    case 706: return D66;
    case 707: return D67;
    case 708: return D68;
    case 709: return D69;
    case 710: return D610;
    case 711: return D611;
    case 712: return D612;
    case 713: return D613;
    case 714: return D614;
    case 715: return D615;
    case 716: return D616;
    case 801: return D71;
    case 806: return D76;
    case 807: return D77;
    case 808: return D78;
    case 809: return D79;
    case 810: return D710;
    case 811: return D711;
    case 812: return D712;
    case 813: return D713;
    case 814: return D714;
    case 815: return D715;
    case 816: return D716;
    default: return 0.0;
    }
}

struct AdjointArgs {
    int64_t n;
    int32_t nt;
    int32_t reserved;
    const double *ts;
    double t0;
    const double *t_end;
    const double *tape;
    int64_t tape_steps;
    int32_t tape_stride;
    int32_t reserved2;
    const uint32_t *n_accepted;
    const uint8_t *status;
    const double *grad_out;
    double *grad_y0;
    double *grad_params;
    drift_potential potential;
    BulgeTable bulge;
};

constexpr int ADJ_THREADS = 128;

template <class Pot>
__device__ __forceinline__ void rhs(const Pot &pot, const double *q, double *k)
{
    k[0] = q[3];
    k[1] = q[4];
    k[2] = q[5];
    pot.force(q[0], q[1], q[2], k[3], k[4], k[5]);
}

// Stage i's cotangent Li through k_i = f(z_i): returns lambda_z.
template <class Jac>
__device__ __forceinline__ void stage_vjp(const Jac &jac, const double *zpos, const double *Li,
                                          double *lz, double *dp)
{
    double jw[3];
    jac.vjp(zpos[0], zpos[1], zpos[2], Li + 3, jw, dp);
    lz[0] = jw[0];
    lz[1] = jw[1];
    lz[2] = jw[2];
    lz[3] = Li[0];
    lz[4] = Li[1];
    lz[5] = Li[2];
}

// One step's stages from y: stage positions Z[i] (i = 1..13, and 14..16
// when `dense`), stage derivatives K, and the new state.
template <class Pot>
__device__ __forceinline__ void recompute_step(const Pot &pot, const double *y, double h, bool dense,
                                               double (&K)[17][6], double (&Z)[17][3], double *ynew)
{
    double z[6];
#pragma unroll
    for (int c = 0; c < 3; c++) Z[1][c] = y[c];
    rhs(pot, y, K[1]);
#pragma unroll
    for (int i = 2; i <= 12; i++) {
#pragma unroll
        for (int c = 0; c < 6; c++) {
            double acc = 0.0;
#pragma unroll
            for (int j = 1; j < i; j++)
                if (acoef(i, j) != 0.0) acc += acoef(i, j) * K[j][c];
            z[c] = y[c] + h * acc;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) Z[i][c] = z[c];
        rhs(pot, z, K[i]);
    }
#pragma unroll
    for (int c = 0; c < 6; c++) {
        double acc = 0.0;
#pragma unroll
        for (int j = 1; j <= 12; j++)
            if (bcoef(j) != 0.0) acc += bcoef(j) * K[j][c];
        ynew[c] = y[c] + h * acc;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) Z[13][c] = ynew[c];
    if (dense) {
        rhs(pot, ynew, K[13]);
#pragma unroll
        for (int i = 14; i <= 16; i++) {
#pragma unroll
            for (int c = 0; c < 6; c++) {
                double acc = 0.0;
#pragma unroll
                for (int j = 1; j < i; j++)
                    if (acoef(i, j) != 0.0) acc += acoef(i, j) * K[j][c];
                z[c] = y[c] + h * acc;
            }
#pragma unroll
            for (int c = 0; c < 3; c++) Z[i][c] = z[c];
            rhs(pot, z, K[i]);
        }
    }
}

#ifndef DRIFT_ADJ_MIN_BLOCKS
#define DRIFT_ADJ_MIN_BLOCKS 1
#endif

template <class Pot, class Jac>
__global__ void __launch_bounds__(ADJ_THREADS, DRIFT_ADJ_MIN_BLOCKS) adjoint_kernel(const __grid_constant__ AdjointArgs a)
{
    __shared__ __align__(16) double table[BOVY_SMEM_DOUBLES];
    if (std::is_same<Pot, Bovy>::value) {
        stage_bovy_tables(table, a.bulge);
        __syncthreads();
    }
    const Pot pot(a.potential, table);
    const Jac jac(a.potential, table);

    for (int64_t pid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pid < a.n;
         pid += (int64_t)gridDim.x * blockDim.x) {
        Grid grid;
        grid.ts = a.ts;
        grid.t0 = a.t0;
        grid.nt = a.nt;
        grid.t_end = a.ts ? 0.0 : a.t_end[pid];
        const int64_t nacc = a.n_accepted[pid];
        const bool ok = (a.status ? a.status[pid] == DRIFT_PARTICLE_OK : true) && nacc >= 1 &&
                        nacc <= a.tape_steps;
        double *gy = a.grad_y0 + pid * 6;
        double *gp = a.grad_params ? a.grad_params + pid * DRIFT_ADJOINT_MAX_PARAMS : nullptr;
        if (!ok) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
            for (int i = 0; i < 6; i++) gy[i] = nan;
            if (gp)
                for (int i = 0; i < DRIFT_ADJOINT_MAX_PARAMS; i++) gp[i] = nan;
            continue;
        }
        const double pos_neg = custom_sign(1.0, grid.at(grid.nt - 1) - grid.at(0));
        double ly[6] = {0, 0, 0, 0, 0, 0};   // cotangent of y_{n+1}
        double lk1[6] = {0, 0, 0, 0, 0, 0};  // cotangent of f(y_{n+1}) (the next step's k_1)
        double dp[DRIFT_ADJOINT_MAX_PARAMS] = {0, 0, 0, 0, 0, 0};
        int32_t khi = grid.nt - 1;  // highest sample not yet propagated
        double y0[6];                // the first step's initial state

        // Reverse of one accepted step that started at (t_old, y) with size h.
        auto reverse_step = [&](const double *y, double t_old, double h) {
            // Samples of this step: t_old <= t_k (in the direction of
            // integration), above the samples of later steps.
            int32_t klo = khi;
            while (klo >= 1 && !(pos_neg * grid.at(klo) < pos_neg * t_old)) klo--;
            const bool dense = khi > klo;

            double K[17][6];
            double Z[17][3];
            double ynew_unused[6];
            recompute_step(pot, y, h, dense, K, Z, ynew_unused);

            double L[17][6];
#pragma unroll
            for (int i = 1; i <= 16; i++)
#pragma unroll
                for (int c = 0; c < 6; c++) L[i][c] = 0.0;
            double lynew[6], lyn[6];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                lynew[c] = ly[c];
                lyn[c] = 0.0;
                L[13][c] = lk1[c];
            }
            if (dense) {
                for (int32_t k = klo + 1; k <= khi; k++) {
                    const double sc = (grid.at(k) - t_old) / h;
                    const double s1 = 1.0 - sc;
                    const double c2 = sc, c3 = sc * s1, c4 = c3 * sc, c5 = c4 * s1, c6 = c5 * sc,
                                 c7 = c6 * s1, c8 = c7 * sc;
                    const double *g = a.grad_out + ((int64_t)k * a.n + pid) * 6;
#pragma unroll
                    for (int c = 0; c < 6; c++) {
                        const double gc = g[c];
                        // r1 = y, r2 = y_new - y, r3 = h k1 - r2, r4 = r2 - h k13 - r3
                        const double lr4 = c4 * gc;
                        const double lr3 = c3 * gc - lr4;
                        const double lr2 = c2 * gc + lr4 - lr3;
                        lyn[c] += gc - lr2;
                        lynew[c] += lr2;
                        L[1][c] += h * lr3;
                        L[13][c] -= h * lr4;
                        const double lr5 = h * c5 * gc, lr6 = h * c6 * gc, lr7 = h * c7 * gc,
                                     lr8 = h * c8 * gc;
#pragma unroll
                        for (int j = 1; j <= 16; j++) {
                            if (dcoef(5, j) != 0.0 || dcoef(6, j) != 0.0 || dcoef(7, j) != 0.0 ||
                                dcoef(8, j) != 0.0)
                                L[j][c] += dcoef(5, j) * lr5 + dcoef(6, j) * lr6 + dcoef(7, j) * lr7 +
                                           dcoef(8, j) * lr8;
                        }
                    }
                }
                // dense stages 16, 15, 14
#pragma unroll
                for (int i = 16; i >= 14; i--) {
                    double lz[6];
                    stage_vjp(jac, Z[i], L[i], lz, dp);
#pragma unroll
                    for (int c = 0; c < 6; c++) {
                        lyn[c] += lz[c];
#pragma unroll
                        for (int j = 1; j < i; j++)
                            if (acoef(i, j) != 0.0) L[j][c] += h * acoef(i, j) * lz[c];
                    }
                }
            }
            // FSAL stage: k13 = f(y_new)
            {
                double lz[6];
                stage_vjp(jac, Z[13], L[13], lz, dp);
#pragma unroll
                for (int c = 0; c < 6; c++) lynew[c] += lz[c];
            }
            // y_new = y + h sum b_j k_j
#pragma unroll
            for (int c = 0; c < 6; c++) {
                lyn[c] += lynew[c];
#pragma unroll
                for (int j = 1; j <= 12; j++)
                    if (bcoef(j) != 0.0) L[j][c] += h * bcoef(j) * lynew[c];
            }
            // stages 12 .. 2
#pragma unroll
            for (int i = 12; i >= 2; i--) {
                double lz[6];
                stage_vjp(jac, Z[i], L[i], lz, dp);
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    lyn[c] += lz[c];
#pragma unroll
                    for (int j = 1; j < i; j++)
                        if (acoef(i, j) != 0.0) L[j][c] += h * acoef(i, j) * lz[c];
                }
            }
#pragma unroll
            for (int c = 0; c < 6; c++) {
                ly[c] = lyn[c];
                lk1[c] = L[1][c];
            }
            khi = klo;
        };

        auto load_row = [](const double *row, double &t, double &h, double *y) {
            const double2 *r = reinterpret_cast<const double2 *>(row);
            double2 v0 = r[0], v1 = r[1], v2 = r[2], v3 = r[3];
            t = v0.x;
            h = v0.y;
            y[0] = v1.x;
            y[1] = v1.y;
            y[2] = v2.x;
            y[3] = v2.y;
            y[4] = v3.x;
            y[5] = v3.y;
        };

        if (a.tape_stride <= 1) {
            // every step is a row (t_old, h, y_old)
            const double *tape = a.tape + pid * a.tape_steps * 8;
            for (int64_t s = nacc - 1; s >= 0; --s) {
                double t_old, h;
                load_row(tape + s * 8, t_old, h, y0);
                reverse_step(y0, t_old, h);
            }
        } else {
            // checkpoints every m steps: recompute the states between them
            const int64_t m = a.tape_stride;
            const int64_t ncp = (a.tape_steps + m - 1) / m;
            const double *block = a.tape + pid * (ncp * 8 + ((a.tape_steps + 1) & ~int64_t(1)));
            const double *hs = block + ncp * 8;
            double ys[DRIFT_MAX_TAPE_STRIDE][6];
            double tt[DRIFT_MAX_TAPE_STRIDE];
            for (int64_t cp = (nacc - 1) / m; cp >= 0; --cp) {
                const int64_t j0 = cp * m;
                const int cnt = (int)min(m, nacc - j0);
                double h0;
                load_row(block + cp * 8, tt[0], h0, ys[0]);
                for (int q = 0; q + 1 < cnt; q++) {
                    double K[17][6];
                    double Z[17][3];
                    const double hq = hs[j0 + q];
                    recompute_step(pot, ys[q], hq, false, K, Z, ys[q + 1]);
                    tt[q + 1] = tt[q] + hq;
                }
                for (int q = cnt - 1; q >= 0; q--) reverse_step(ys[q], tt[q], hs[j0 + q]);
                if (cp == 0)
                    for (int c = 0; c < 6; c++) y0[c] = ys[0][c];
            }
        }
        // k_1 of the first step is f(y0) (begin); sample 0 is y0 itself.
        {
            double lz[6];
            stage_vjp(jac, y0, lk1, lz, dp);
            const double *g0 = a.grad_out + pid * 6;
#pragma unroll
            for (int c = 0; c < 6; c++) gy[c] = ly[c] + lz[c] + g0[c];
        }
        if (gp)
#pragma unroll
            for (int i = 0; i < DRIFT_ADJOINT_MAX_PARAMS; i++) gp[i] = dp[i];
    }
}

cudaError_t launch(const AdjointArgs &a, int grid, int block, cudaStream_t s)
{
    switch (a.potential.kind) {
    case DRIFT_POT_KEPLER: adjoint_kernel<KeplerGalpy, KeplerJac><<<grid, block, 0, s>>>(a); break;
    case DRIFT_POT_KEPLER_CARTESIAN:
        adjoint_kernel<KeplerCartesian, KeplerJac><<<grid, block, 0, s>>>(a);
        break;
    case DRIFT_POT_PLUMMER: adjoint_kernel<Plummer, PlummerJac><<<grid, block, 0, s>>>(a); break;
    case DRIFT_POT_BOVY: adjoint_kernel<Bovy, BovyJac><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace adjoint
}  // namespace drift

extern "C" int drift_integrate_adjoint(const drift_adjoint_launch *A, void *stream)
{
    drift::TraceRange trace("drift integrate adjoint");
    if (!A) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "adjoint launch is NULL");
    if (A->method != DRIFT_DOP853)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "the adjoint supports DOP853");
    const int k = A->potential.kind;
    if (k < DRIFT_POT_KEPLER || k > DRIFT_POT_KEPLER_CARTESIAN)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "unknown potential kind");
    if (A->n < 1 || A->nt < 2 || A->nt > INT32_MAX - 1)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "n must be >= 1 and nt in [2, 2^31 - 2]");
    if (!A->ts && !A->t_end)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "either ts or t_end is required");
    if (!A->tape || A->tape_steps < 1 || !A->n_accepted || !A->grad_out || !A->grad_y0)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT,
                                   "tape, tape_steps, n_accepted, grad_out and grad_y0 are required");
    if (reinterpret_cast<uintptr_t>(A->tape) % 16)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "the tape must be 16-byte aligned");
    if (A->tape_stride > DRIFT_MAX_TAPE_STRIDE)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "tape_stride must be at most 16");
    if (A->block_size != 0 && (A->block_size < 32 || A->block_size > drift::adjoint::ADJ_THREADS ||
                               A->block_size % 32))
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT,
                                   "block_size must be 0 or a multiple of 32 in [32, 128]");
    drift::adjoint::AdjointArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = A->n;
    a.nt = (int32_t)A->nt;
    a.ts = A->ts;
    a.t0 = A->t0;
    a.t_end = A->t_end;
    a.tape = A->tape;
    a.tape_steps = A->tape_steps;
    a.tape_stride = A->tape_stride;
    a.n_accepted = A->n_accepted;
    a.status = A->status;
    a.grad_out = A->grad_out;
    a.grad_y0 = A->grad_y0;
    a.grad_params = A->grad_params;
    a.potential = A->potential;
    if (k == DRIFT_POT_BOVY) drift::fill_bulge_table(1.5 - 0.5 * A->potential.bulge_alpha, &a.bulge);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    // Default block: the largest of 128, 64, 32 threads that still gives
    // every SM two blocks, so small particle counts spread over the GPU.
    int block = A->block_size;
    if (!block) {
        block = drift::adjoint::ADJ_THREADS;
        while (block > 32 && (A->n + block - 1) / block < 2 * (int64_t)sms) block /= 2;
    }
    const int64_t blocks = std::min<int64_t>((A->n + block - 1) / block, (int64_t)sms * 64);
    cudaError_t e = drift::adjoint::launch(a, (int)blocks, block, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess)
        return drift_internal_fail(DRIFT_ERROR_CUDA, (std::string("adjoint kernel launch: ") +
                                                      cudaGetErrorString(e)).c_str());
    return DRIFT_SUCCESS;
}
