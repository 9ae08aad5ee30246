// dare_assembly3.cu -- assembly of 3-D grids (DDT + TVD convection +
// diffusion + boundary folding), staged through shared memory.
//
// The composed functor of the reference's time loops
//     mb  = ddt(field)                 DDT.inl:39-81
//     mb += div(TVD(vel) * field)      TVD_Cartesian.inl:185-261, Divergence_Cartesian.inl:139-207
//     mb -= div(D, grad(mb))           Gradient_Cartesian.inl:37-58, Divergence_Cartesian.inl:90-96
//     fold W,E,S,N,B,T boundary faces  counter_diffusion1D.cpp:123-146
// reduces, per direction d with lower / upper face velocities vl, vu, face
// diffusivities Dl, Du, area A = V/dx_d and 1/dx_d = dn, to
//     W_d = -w0 A max(vl, 0) - w0 A dn Dl
//     E_d =  w0 A min(vu, 0) - w0 A dn Du
//     C  += w0 A (max(vu, 0) - min(vl, 0)) + w0 A dn (Dl + Du)
//     rhs += (1 + sum_t w_t) A (rr_u - rr_l),  rr = -0.5 psi(r) (phi_D - phi_U) v
// with C = V/dt and rhs = V/dt phi_old from DDT (w = the Divergence time
// scheme's weights).  These are the same coefficients as the per-cell
// functor; only the rounding differs (FMA contraction, the limiter in the
// division-light forms below), within 1e-13 relative of the CPU path.
//
// Flux limiters as psi(r) * den, with r = num / den, num = phi_U - phi_UU,
// den = phi_D - phi_U (FluxLimiter.h:41-173):
//   van Leer  (r + |r|) / (1 + |r|) * den = 2 num den / (num + den) when num
//             and den have the same sign, else 0 (one division instead of two,
//             by Newton-Raphson, div_nr; r = 0/0 -> 0 and r = +-inf -> 2 * 0 = 0
//             as in the r form)
//   MINMOD    max(0, min(r, 1)) * den = |num| < |den| ? num : den when num and
//             den have the same sign, else 0 (no division)
//   CDS, UPWIND  den, 0
//   VANALBADA keeps the r form: r = +-inf gives NaN there, as in the reference.
//
// Work decomposition: a block owns a tile of 32 cells along k (one warp per
// row) by 8 rows along j and marches along i over a run of planes.  Every
// plane is staged by cp.async into one slot of a 5-deep ring: phi with its
// 2-cell j/k halo (12 x 36), phi_old, and the face arrays of the tile (x
// faces above the cells, 9 rows of y faces, 33 columns of z faces).  Two
// planes are in flight while one is computed, so HBM latency hides behind
// the arithmetic.  The x line phi(i-2..i+2) of a cell stays in registers.
// Each TVD face is evaluated once: a cell evaluates its upper faces E, N, T;
// W is its own E of the previous plane, S the N face of the row below
// (shared memory; row 0 evaluates S), B the T face of the lane below (warp
// shuffle; lane 0 evaluates B).
//
// Algorithmic traffic per cell (constant D, face velocities): phi, phi_old
// and three face velocities read (40 B), 7 diagonals, rhs and x0 written
// (72 B): 112 B; face D adds 24 B.
#include "dare_assembly.cuh"
#include "dare_march.cuh"

namespace dare_gpu {

constexpr int kA3K = 32, kA3J = 8;                    // tile: cells along k x rows along j
constexpr int kA3Ring = 5;                            // staged planes
constexpr int kA3PW = kA3K + 4, kA3PH = kA3J + 4;     // phi tile with its 2-cell halo
constexpr int kA3Phi = kA3PW * kA3PH;                 // 432
constexpr int kA3Cell = kA3K * kA3J;                  // 256
constexpr int kA3FY = (kA3J + 1) * kA3K;              // 288: y faces of rows j0 .. j0+8
constexpr int kA3FZW = kA3K + 1;
constexpr int kA3FZ = kA3J * kA3FZW;                  // 264: z faces k0 .. k0+32
// offsets inside one stage (doubles)
constexpr int kOffPO = kA3Phi;
constexpr int kOffVX = kOffPO + kA3Cell;
constexpr int kOffVY = kOffVX + kA3Cell;
constexpr int kOffVZ = kOffVY + kA3FY;
constexpr int kOffDX = kOffVZ + kA3FZ;
constexpr int kOffDY = kOffDX + kA3Cell;
constexpr int kOffDZ = kOffDY + kA3FY;
template <bool FD>
__host__ __device__ constexpr int a3_stage() {
    return FD ? kOffDZ + kA3FZ : kOffDX;
}

// Scalars of the reduced coefficient formulas (host-evaluated).
struct A3Params {
    double tt;          // V / dt (0 without DDT)
    int ddt;
    int conv;           // 0 none, 1 constant velocity, 2 face velocities
    double vel[3];
    double cA[3];       // w0 A_d (convection coefficients)
    double rA[3];       // (1 + sum_t w_t) A_d (deferred-correction rhs)
    int diff;           // 0 none, 1 scalar D, 2 face D
    double kD[3];       // scalar D: w0 A_d dn_d D;  face D: w0 A_d dn_d
    int bc_type[6];
    double bc_value[6];
    int64_t dstride;
    const double* face_vel[3];
    const double* face_D[3];
    int acc;            // add to the coefficients already in the system
    int fold;           // fold the boundary faces at the end
    int xint;           // x ends shared with a neighbouring slab (bit 0 low, bit 1 high): not folded
};

// a / b for normal, finite b by Newton-Raphson refinement of the hardware
// reciprocal estimate (PTX rcp.approx.ftz.f64): each step y <- y + y (1 - b y)
// squares the relative error e of y, and the residual correction of the
// quotient, q + y (a - b q) (Markstein's correction), squares it once more,
// so an estimate with e <= 2^-7 already ends below 2^-56.  The result is
// within an ulp or two of the IEEE quotient, without the IEEE division's
// special-case branches (the assembly parity tests hold it to 1e-13 of the
// CPU path's IEEE divisions, also on fields spanning twelve decades).  Used
// by the van Leer limiter, where b = num + den is a sum of two same-signed
// differences of field values.
__device__ __forceinline__ double div_nr(double a, double b) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    const double q = a * y;
    const double r = fma(-b, q, a);
    return fma(r, y, q);
}

template <int LIM>
__device__ __forceinline__ double face_flux(double a, double b, double c, double d, double v) {
    const bool vp = v >= 0.;
    const double pUU = vp ? a : d, pU = vp ? b : c, pD = vp ? c : b;
    const double num = pU - pUU, den = pD - pU;
    // num and den of the same sign (r > 0); a product below the smallest
    // normal reads as r <= 0, which changes rr by less than that product
    const bool same = num * den > 0.;
    if constexpr (LIM == DARE_LIMITER_CDS) {
        return (-0.5 * den) * v;
    } else if constexpr (LIM == DARE_LIMITER_UPWIND) {
        return 0.;
    } else if constexpr (LIM == DARE_LIMITER_MINMOD) {
        const double pd = same ? (fabs(num) < fabs(den) ? num : den) : 0.;
        return (-0.5 * pd) * v;
    } else if constexpr (LIM == DARE_LIMITER_VANLEER) {
        // -0.5 * (2 num den / (num + den)) * v; den / (num + den) lies in (0, 1)
        return same ? -(num * div_nr(den, num + den)) * v : 0.;
    } else {
        const double psi = limiter_value(LIM, num / den);
        return ((-0.5 * psi) * den) * v;
    }
}

// In-plane offsets and validity of the elements a thread stages, fixed for
// the block's tile: index e of an array of the stage maps to row e / width,
// column e % width of the tile.
struct A3Copy {
    int off;     // in-plane element offset in the source array (< 0: zero fill)
    int sm;      // element in the stage
};

template <int LIM, bool FD, bool PAIR>
__global__ void __launch_bounds__(256, FD ? 2 : 3)
    k_assemble3(GridDev g, A3Params a, const double* __restrict__ phi, const double* __restrict__ phi_old,
                double* __restrict__ diag, double* __restrict__ rhs_out, double* __restrict__ x0, int planes,
                int ibase, int iend) {
    constexpr int STAGE = a3_stage<FD>();
    extern __shared__ __align__(16) double sm3[];
    __shared__ double rrN_s[2][kA3J][kA3K];
    const int lane = threadIdx.x, ty = threadIdx.y, tid = lane + kA3K * ty;
    const int n1 = g.n[1], n2 = g.n[2];
    const int gn1 = g.gn[1], gn2 = g.gn[2];
    const int og0 = g.og[0], og1 = g.og[1], og2 = g.og[2];
    const int k0 = blockIdx.x * kA3K, j0 = blockIdx.y * kA3J;
    const int kk = k0 + lane, jj = j0 + ty;
    const bool active = kk < n2 && jj < n1;
    const int i0 = ibase + blockIdx.z * planes;   // this block's run of the planes ibase .. iend - 1
    const int i1 = min(i0 + planes, iend);
    const int P = (i1 - i0) + 4;                    // staged planes i0-2 .. i1+1
    const int64_t gplane = (int64_t)gn1 * gn2;
    const int64_t xplane = (int64_t)n1 * n2, yplane = (int64_t)(n1 + 1) * n2, zplane = (int64_t)n1 * (n2 + 1);
    const bool fvel = a.conv == 2;

    // ---- the elements this thread stages (offsets within a plane) ----------
    A3Copy cph[2], cpo, cy[2], cz[2];
    for (int h = 0; h < 2; h++) {
        const int e = tid + h * 256;
        cph[h].sm = e;
        cph[h].off = -1;
        if (e < kA3Phi) {
            const int j = j0 - 2 + e / kA3PW, k = k0 - 2 + e % kA3PW;
            if (j + og1 >= 0 && j + og1 < gn1 && k + og2 >= 0 && k + og2 < gn2) cph[h].off = (j + og1) * gn2 + k + og2;
        }
        cy[h].sm = kOffVY + e;
        cy[h].off = -1;
        if (e < kA3FY) {
            int f = j0 + e / kA3K;
            const int k = k0 + e % kA3K;
            if (f == n1 && g.periodic[1]) f = 0;
            if (f <= n1 && k < n2) cy[h].off = f * n2 + k;
        }
        cz[h].sm = kOffVZ + e;
        cz[h].off = -1;
        if (e < kA3FZ) {
            const int j = j0 + e / kA3FZW;
            int f = k0 + e % kA3FZW;
            if (f == n2 && g.periodic[2]) f = 0;
            if (j < n1 && f <= n2) cz[h].off = j * (n2 + 1) + f;
        }
    }
    cpo.sm = tid;
    cpo.off = active ? jj * n2 + kk : -1;
    const int cell_gh = (jj + og1) * gn2 + kk + og2;     // the cell's ghosted in-plane offset (active cells)

    // PAIR (even n2 and ghost width, 16-byte aligned arrays): the same
    // elements staged as 16-byte pairs of cells.  Each thread: one pair of the
    // phi tile (216 pairs), one pair of phi_old (threads 0-127) or of the x
    // faces (128-255), one pair of the y faces (0-143); the z faces (rows of
    // n2 + 1) stay single.  The shared-memory layout is the one above.
    A3Copy pph{-1, 0}, pov{-1, 0}, pvy{-1, 0}, pdx{-1, 0};
    if constexpr (PAIR) {
        if (tid < kA3Phi / 2) {
            const int row = tid / (kA3PW / 2), col = 2 * (tid - row * (kA3PW / 2));
            pph.sm = row * kA3PW + col;
            const int j = j0 - 2 + row, k = k0 - 2 + col;
            if (j + og1 >= 0 && j + og1 < gn1 && k + og2 >= 0 && k + og2 < gn2) pph.off = (j + og1) * gn2 + k + og2;
        }
        {
            const int t2 = tid & 127, row = t2 >> 4, c2 = 2 * (t2 & 15);
            const int pj = j0 + row, pk = k0 + c2;
            const bool act = pj < n1 && pk < n2;
            if (tid < 128) {   // phi_old (ghosted) and, with face D, the x faces of D
                pov.sm = kOffPO + row * kA3K + c2;
                pov.off = act ? (pj + og1) * gn2 + pk + og2 : -1;
                pdx.sm = kOffDX + row * kA3K + c2;
                pdx.off = act ? pj * n2 + pk : -1;
            } else {           // the x faces of the velocity
                pov.sm = kOffVX + row * kA3K + c2;
                pov.off = act ? pj * n2 + pk : -1;
            }
        }
        if (tid < kA3FY / 2) {
            const int row = tid >> 4, c2 = 2 * (tid & 15);
            int f = j0 + row;
            const int k = k0 + c2;
            if (f == n1 && g.periodic[1]) f = 0;
            pvy.sm = kOffVY + row * kA3K + c2;
            pvy.off = (f <= n1 && k < n2) ? f * n2 + k : -1;
        }
    }

    auto slot = [&](int s) { return sm3 + (size_t)(s % kA3Ring) * STAGE; };
    // stage sequence index s: plane i0 - 2 + s
    auto stage = [&](int s) {
        if (s >= P) return;
        const int p = i0 - 2 + s;
        double* sb = slot(s);
        const double* src = phi + (int64_t)(p + og0) * gplane;
        if constexpr (PAIR) {
            if (tid < kA3Phi / 2) cp_async<16>(sb + pph.sm, src + (pph.off < 0 ? 0 : pph.off), pph.off >= 0);
            if (p < i0 || p >= i1) return;                // halo planes: phi only
            const int pu = upper_face(g, 0, p);
            if (tid < 128)
                cp_async<16>(sb + pov.sm, phi_old + (int64_t)(p + og0) * gplane + (pov.off < 0 ? 0 : pov.off),
                             pov.off >= 0);
            if (fvel) {
                if (tid >= 128)
                    cp_async<16>(sb + pov.sm, a.face_vel[0] + pu * xplane + (pov.off < 0 ? 0 : pov.off), pov.off >= 0);
                if (tid < kA3FY / 2)
                    cp_async<16>(sb + pvy.sm, a.face_vel[1] + p * yplane + (pvy.off < 0 ? 0 : pvy.off), pvy.off >= 0);
#pragma unroll
                for (int h = 0; h < 2; h++)
                    if (cz[h].sm < kOffVZ + kA3FZ)
                        cp_async<8>(sb + cz[h].sm, a.face_vel[2] + p * zplane + (cz[h].off < 0 ? 0 : cz[h].off),
                                    cz[h].off >= 0);
            }
            if constexpr (FD) {
                constexpr int dy = kOffDY - kOffVY, dz = kOffDZ - kOffVZ;
                if (tid < 128)
                    cp_async<16>(sb + pdx.sm, a.face_D[0] + pu * xplane + (pdx.off < 0 ? 0 : pdx.off), pdx.off >= 0);
                if (tid < kA3FY / 2)
                    cp_async<16>(sb + pvy.sm + dy, a.face_D[1] + p * yplane + (pvy.off < 0 ? 0 : pvy.off), pvy.off >= 0);
#pragma unroll
                for (int h = 0; h < 2; h++)
                    if (cz[h].sm < kOffVZ + kA3FZ)
                        cp_async<8>(sb + cz[h].sm + dz, a.face_D[2] + p * zplane + (cz[h].off < 0 ? 0 : cz[h].off),
                                    cz[h].off >= 0);
            }
        } else {
#pragma unroll
            for (int h = 0; h < 2; h++)
                if (cph[h].sm < kA3Phi) cp_async<8>(sb + cph[h].sm, src + (cph[h].off < 0 ? 0 : cph[h].off), cph[h].off >= 0);
            if (p < i0 || p >= i1) return;                    // halo planes: phi only
            cp_async<8>(sb + kOffPO + tid, phi_old + (int64_t)(p + og0) * gplane + (cpo.off < 0 ? 0 : cell_gh),
                        cpo.off >= 0);
            const int pu = upper_face(g, 0, p);
            if (fvel) {
                cp_async<8>(sb + kOffVX + tid, a.face_vel[0] + pu * xplane + (cpo.off < 0 ? 0 : cpo.off), cpo.off >= 0);
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    if (cy[h].sm < kOffVY + kA3FY)
                        cp_async<8>(sb + cy[h].sm, a.face_vel[1] + p * yplane + (cy[h].off < 0 ? 0 : cy[h].off),
                                    cy[h].off >= 0);
                    if (cz[h].sm < kOffVZ + kA3FZ)
                        cp_async<8>(sb + cz[h].sm, a.face_vel[2] + p * zplane + (cz[h].off < 0 ? 0 : cz[h].off),
                                    cz[h].off >= 0);
                }
            }
            if constexpr (FD) {
                constexpr int dy = kOffDY - kOffVY, dz = kOffDZ - kOffVZ;
                cp_async<8>(sb + kOffDX + tid, a.face_D[0] + pu * xplane + (cpo.off < 0 ? 0 : cpo.off), cpo.off >= 0);
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    if (cy[h].sm < kOffVY + kA3FY)
                        cp_async<8>(sb + cy[h].sm + dy, a.face_D[1] + p * yplane + (cy[h].off < 0 ? 0 : cy[h].off),
                                    cy[h].off >= 0);
                    if (cz[h].sm < kOffVZ + kA3FZ)
                        cp_async<8>(sb + cz[h].sm + dz, a.face_D[2] + p * zplane + (cz[h].off < 0 ? 0 : cz[h].off),
                                    cz[h].off >= 0);
                }
            }
        }
    };

    const int cen = (ty + 2) * kA3PW + lane + 2;          // the cell in the phi tile
    // prologue: planes i0-2 .. i0+1 give the x line and the first W face
    for (int s = 0; s < 4; s++) {
        stage(s);
        cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();
    double w0 = slot(0)[cen], w1 = slot(1)[cen], w2 = slot(2)[cen], w3 = slot(3)[cen], w4 = 0.;
    const int64_t xlo = (int64_t)i0 * xplane + (cpo.off < 0 ? 0 : cpo.off);
    double vW = a.conv == 1 ? a.vel[0] : (fvel ? a.face_vel[0][xlo] : 0.);
    double DW = 0.;
    if constexpr (FD) DW = a.face_D[0][xlo];
    double rrW = a.conv ? face_flux<LIM>(w0, w1, w2, w3, vW) : 0.;
    __syncthreads();                                      // slots 0 and 1 are reused below
    stage(4);
    cp_async_commit();
    stage(5);
    cp_async_commit();

    int64_t c = (int64_t)i0 * xplane + (int64_t)jj * n2 + kk;
    for (int i = i0; i < i1; i++) {
        const int t = i - i0;
        stage(t + 6);                                     // into the slot of plane i - 1
        cp_async_commit();
        cp_async_wait<2>();                               // planes up to i + 2 have landed
        __syncthreads();
        const double* sb = slot(t + 2);
        w4 = slot(t + 4)[cen];
        const int buf = t & 1;
        double cC = a.ddt ? a.tt : 0.;
        double rhs = a.ddt ? a.tt * sb[kOffPO + tid] : 0.;
        double cW = 0., cE = 0., cS = 0., cN = 0., cB = 0., cT = 0.;
        double vE = 0., vS = 0., vN = 0., vB = 0., vT = 0.;
        if (a.conv) {
            if (fvel) {
                vE = sb[kOffVX + tid];
                vS = sb[kOffVY + ty * kA3K + lane];
                vN = sb[kOffVY + (ty + 1) * kA3K + lane];
                vB = sb[kOffVZ + ty * kA3FZW + lane];
                vT = sb[kOffVZ + ty * kA3FZW + lane + 1];
            } else {
                vE = a.vel[0];
                vS = vN = a.vel[1];
                vB = vT = a.vel[2];
            }
            const double ym1 = sb[cen - kA3PW], yp1 = sb[cen + kA3PW], yp2 = sb[cen + 2 * kA3PW];
            const double zm1 = sb[cen - 1], zp1 = sb[cen + 1], zp2 = sb[cen + 2];
            const double rrE = face_flux<LIM>(w1, w2, w3, w4, vE);
            const double rrN = face_flux<LIM>(ym1, w2, yp1, yp2, vN);
            const double rrT = face_flux<LIM>(zm1, w2, zp1, zp2, vT);
            rrN_s[buf][ty][lane] = rrN;
            double rrB = __shfl_up_sync(0xFFFFFFFFu, rrT, 1);
            if (lane == 0) rrB = face_flux<LIM>(sb[cen - 2], zm1, w2, zp1, vB);
            double rrS = 0.;
            if (ty == 0) rrS = face_flux<LIM>(sb[cen - 2 * kA3PW], ym1, w2, yp1, vS);
            __syncthreads();
            if (ty > 0) rrS = rrN_s[buf][ty - 1][lane];
            cW = -a.cA[0] * fmax(vW, 0.);
            cE = a.cA[0] * fmin(vE, 0.);
            cS = -a.cA[1] * fmax(vS, 0.);
            cN = a.cA[1] * fmin(vN, 0.);
            cB = -a.cA[2] * fmax(vB, 0.);
            cT = a.cA[2] * fmin(vT, 0.);
            cC += a.cA[0] * (fmax(vE, 0.) - fmin(vW, 0.)) + a.cA[1] * (fmax(vN, 0.) - fmin(vS, 0.)) +
                  a.cA[2] * (fmax(vT, 0.) - fmin(vB, 0.));
            rhs += a.rA[0] * (rrE - rrW) + a.rA[1] * (rrN - rrS) + a.rA[2] * (rrT - rrB);
            rrW = rrE;
            vW = vE;
        }
        if (a.diff == 1) {
            cW -= a.kD[0];
            cE -= a.kD[0];
            cS -= a.kD[1];
            cN -= a.kD[1];
            cB -= a.kD[2];
            cT -= a.kD[2];
            cC += 2. * (a.kD[0] + a.kD[1] + a.kD[2]);
        }
        if constexpr (FD) {
            const double DE = sb[kOffDX + tid];
            const double DS = sb[kOffDY + ty * kA3K + lane], DN = sb[kOffDY + (ty + 1) * kA3K + lane];
            const double DB = sb[kOffDZ + ty * kA3FZW + lane], DT = sb[kOffDZ + ty * kA3FZW + lane + 1];
            cW -= a.kD[0] * DW;
            cE -= a.kD[0] * DE;
            cS -= a.kD[1] * DS;
            cN -= a.kD[1] * DN;
            cB -= a.kD[2] * DB;
            cT -= a.kD[2] * DT;
            cC += a.kD[0] * (DW + DE) + a.kD[1] * (DS + DN) + a.kD[2] * (DB + DT);
            DW = DE;
        }
        if (active) {
            double coef[7] = {cC, cW, cE, cS, cN, cB, cT};
            if (a.acc) {                                  // a term added to an earlier one
#pragma unroll
                for (int p = 0; p < 7; p++) coef[p] += diag[p * a.dstride + c];
                rhs += rhs_out[c];
            }
            const int idx[3] = {i, jj, kk};
#pragma unroll
            for (int d = 0; d < 3; d++) {                 // boundary folding
                if (g.periodic[d] || !a.fold) continue;
#pragma unroll
                for (int side = 0; side < 2; side++) {
                    const int face = 2 * d + 1 + side;
                    const bool on_boundary = side == 0 ? (idx[d] == 0) : (idx[d] == g.n[d] - 1);
                    if (!on_boundary || (d == 0 && ((a.xint >> side) & 1))) continue;
                    const double X = coef[face];
                    if (a.bc_type[face - 1] == DARE_BC_DIRICHLET) {
                        coef[0] -= X;
                        rhs -= 2. * a.bc_value[face - 1] * X;
                    } else {
                        coef[0] += X;
                    }
                    coef[face] = 0.;
                }
            }
#pragma unroll
            for (int p = 0; p < 7; p++) diag[p * a.dstride + c] = coef[p];
            rhs_out[c] = rhs;
            x0[c] = w2;
        }
        w0 = w1;
        w1 = w2;
        w2 = w3;
        w3 = w4;
        c += xplane;
        __syncthreads();                                  // the slot of plane i is free for plane i + 5
    }
    cp_async_wait<0>();
}

template <int LIM, bool FD, bool PAIR>
static int launch3_k(dare_ctx* ctx, const GridDev& g, const A3Params& p, const double* phi, const double* phi_old,
                     double* diag, double* rhs, double* x0, int ib, int ie) {
    const size_t smem = (size_t)a3_stage<FD>() * kA3Ring * sizeof(double);
    static int resident = 0;
    if (!resident) {
        DARE_CUDA(ctx, cudaFuncSetAttribute(k_assemble3<LIM, FD, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_assemble3<LIM, FD, PAIR>, kA3K * kA3J, smem) !=
                cudaSuccess ||
            occ < 1)
            occ = 1;
        resident = occ * ctx->num_sms;
    }
    // runs of i-planes sized so the waves of resident blocks come out even;
    // a run re-stages 4 planes of phi (its x halo)
    const int n0 = ie - ib;   // the planes of this launch
    const int gx = (g.n[2] + kA3K - 1) / kA3K, gy = (g.n[1] + kA3J - 1) / kA3J;
    const int64_t units = (int64_t)gx * gy;
    int best = n0;
    int64_t best_cost = INT64_MAX;
    for (int chunks = 1; chunks <= n0; chunks++) {
        const int pl = (n0 + chunks - 1) / chunks;
        if ((n0 + pl - 1) / pl != chunks) continue;
        const int64_t cost = ((units * chunks + resident - 1) / resident) * (pl + 4);
        if (cost < best_cost) {
            best_cost = cost;
            best = pl;
        }
    }
    const dim3 grid(gx, gy, (unsigned)((n0 + best - 1) / best)), block(kA3K, kA3J, 1);
    k_assemble3<LIM, FD, PAIR><<<grid, block, smem, ctx->stream>>>(g, p, phi, phi_old, diag, rhs, x0, best, ib, ie);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// PAIR applies with an even n2 and ghost width (the ghosted rows and the
// tile's first column then start on 16-byte boundaries) and 16-byte aligned
// arrays
template <int LIM, bool FD>
static int launch3_t(dare_ctx* ctx, const GridDev& g, const A3Params& p, const double* phi, const double* phi_old,
                     double* diag, double* rhs, double* x0, int ib, int ie) {
    auto al = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    bool pair = g.n[2] % 2 == 0 && g.og[2] % 2 == 0 && al(phi) && al(phi_old);
    if (p.conv == 2) pair = pair && al(p.face_vel[0]) && al(p.face_vel[1]);
    if (FD) pair = pair && al(p.face_D[0]) && al(p.face_D[1]);
    return pair ? launch3_k<LIM, FD, true>(ctx, g, p, phi, phi_old, diag, rhs, x0, ib, ie)
                : launch3_k<LIM, FD, false>(ctx, g, p, phi, phi_old, diag, rhs, x0, ib, ie);
}

int launch_assemble3(dare_ctx* ctx, const GridDev& g, const AsmParams& a, const double* phi, const double* phi_old,
                     double* diag, double* rhs, double* x0, int ib, int ie) {
    if (ie < 0) ie = g.n[0];
    if (ib < 0 || ib >= ie || ie > g.n[0]) return DARE_OK;   // an empty range
    A3Params p{};
    p.ddt = a.dt > 0.;
    p.tt = a.sgn_ddt * a.tt;
    p.conv = a.convection;
    p.diff = a.diffusion;
    p.acc = a.acc;
    p.fold = a.fold;
    p.xint = a.xint;
    double wsum = 1.;
    for (int t = 1; t <= a.nexp; t++) wsum += a.w[t];
    // the parts' signs enter through their factors: the kernel subtracts the
    // diffusion factors (the fused functor's mb -= div(D grad))
    for (int d = 0; d < 3; d++) {
        p.vel[d] = a.vel[d];
        p.cA[d] = a.sgn_conv * (a.w[0] * g.area[d]);
        p.rA[d] = a.sgn_conv * (wsum * g.area[d]);
        p.kD[d] = -a.sgn_diff * (a.w[0] * g.area[d] * a.dn[d] * (a.diffusion == 1 ? a.D : 1.));
        p.face_vel[d] = a.face_vel[d];
        p.face_D[d] = a.face_D[d];
    }
    for (int f = 0; f < 6; f++) {
        p.bc_type[f] = a.bc_type[f];
        p.bc_value[f] = a.bc_value[f];
    }
    p.dstride = a.dstride;
    const bool fd = a.diffusion == 2;
    switch (a.limiter) {
#define DARE_A3(L)                                                                                   \
    case L:                                                                                          \
        return fd ? launch3_t<L, true>(ctx, g, p, phi, phi_old, diag, rhs, x0, ib, ie)               \
                  : launch3_t<L, false>(ctx, g, p, phi, phi_old, diag, rhs, x0, ib, ie);
        DARE_A3(DARE_LIMITER_CDS)
        DARE_A3(DARE_LIMITER_UPWIND)
        DARE_A3(DARE_LIMITER_VANALBADA)
        DARE_A3(DARE_LIMITER_MINMOD)
        DARE_A3(DARE_LIMITER_VANLEER)
#undef DARE_A3
    }
    return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: bad limiter");
}

}  // namespace dare_gpu
