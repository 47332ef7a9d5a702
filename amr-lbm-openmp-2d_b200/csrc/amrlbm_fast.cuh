// amrlbm_fast.cuh - block geometry with compile-time sizes and exact FP64
// division helpers for the hot kernels.
#pragma once

#include "amrlbm_dev.cuh"

// Pool strides of one block; N > 0 makes every stride a compile-time
// constant (the host computes the same values for any nx = ny = N).
template <int N>
struct Geo {
    int nx, ny, ap, aplane, bplane, cp, cplane, pplane;
    __device__ __forceinline__ explicit Geo(const DevState& s)
        : nx(N ? N : s.nx),
          ny(N ? N : s.ny),
          ap(N ? N + 2 : s.ap),
          aplane(N ? (N + 2) * (N + 2) : s.aplane),
          bplane(N ? N * N : s.bplane),
          cp(N ? ((N + 6 + 3) / 4) * 4 : s.cp),
          cplane(N ? (((N + 4) * (((N + 6 + 3) / 4) * 4) + 15) / 16) * 16 : s.cplane),
          pplane(N ? N * N : s.pplane) {}
    __device__ __forceinline__ size_t a(int b, int q, int x, int y) const {
        return ((size_t)b * 9 + (q - 1)) * aplane + (size_t)(y * ap + x);
    }
    __device__ __forceinline__ size_t bb(int b, int q, int x, int y) const {
        return ((size_t)b * 9 + (q - 1)) * bplane + (size_t)((y - 1) * nx + (x - 1));
    }
    __device__ __forceinline__ size_t c(int b, int x, int y) const {
        return (size_t)b * cplane + (size_t)((y + 1) * cp + (x + 3));
    }
    __device__ __forceinline__ size_t p(int b, int x, int y) const {
        return (size_t)b * pplane + (size_t)((y - 1) * nx + (x - 1));
    }
};

// Exact FP64 division by b given yb = RN(1/b). q = RN(a*yb) is a faithful
// approximation of a/b, the remainder r = a - q*b is exact in one FMA, and
// RN(q + r*yb) is the correctly rounded quotient: Markstein's theorem
// (P. W. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990; Muller et al.,
// Handbook of Floating-Point Arithmetic, ch. 4). The theorem needs a normal
// quotient away from underflow and overflow. Div<false> evaluates the
// formula without a branch, returns the exact signed zero for a zero
// dividend, and ORs into `bad` whether any other quotient fell outside
// [2^-960, 2^1001); a caller that sees `bad` recomputes with Div<true>, plain
// IEEE division. Either way every quotient equals the IEEE one (checked bit
// for bit by amrlbm_selftest_division).
template <bool SAFE>
struct Div {
    unsigned bad = 0;
    __device__ __forceinline__ double operator()(double a, double b, double yb) {
        if (SAFE) return a / b;
        const double q = a * yb;
        const double r = __fma_rn(-q, b, a);
        const double q1 = __fma_rn(r, yb, q);
        const unsigned ha = (unsigned)__double2hiint(a), la = (unsigned)__double2loint(a);
        const bool a0 = ((ha & 0x7fffffffu) | la) == 0u;
        const unsigned e = ((unsigned)__double2hiint(q) >> 20) & 0x7ffu;
        bad |= (unsigned)((e - 63u > 1960u) & !a0);
        return a0 ? q : q1;
    }
    __device__ __forceinline__ double d3(double a) { return (*this)(a, 3.0, 1.0 / 3.0); }
    __device__ __forceinline__ double d6(double a) { return (*this)(a, 6.0, 1.0 / 6.0); }
    __device__ __forceinline__ double d12(double a) { return (*this)(a, 12.0, 1.0 / 12.0); }
    __device__ __forceinline__ double d36(double a) { return (*this)(a, 36.0, 1.0 / 36.0); }
};

// Gradient_ED_AMR (LBM_Subroutines.f90:281-289) from a directional
// derivative functor E(k)
template <class DV, class EF>
__device__ __forceinline__ void gradient_ed_f(DV& dv, EF E, double& Dx, double& Dy) {
    Dx = dv.d3(E(2) - E(4)) + dv.d12(E(6) - E(7) - E(8) + E(9));
    Dy = dv.d3(E(3) - E(5)) + dv.d12(E(6) + E(7) - E(8) - E(9));
}

// Gradient_AMR (LBM_Subroutines.f90:293-312) at one cell; inv_dx = 1/dx (dx
// is a power of two, so the product equals the quotient)
template <class DV, class CF>
__device__ __forceinline__ void gradient_iso_f(DV& dv, double inv_dx, CF Cs, double& DcDx,
                                               double& DcDy) {
    DcDx = (dv.d3(Cs(1, 0) - Cs(-1, 0)) + dv.d12(Cs(1, 1) + Cs(1, -1) - Cs(-1, 1) - Cs(-1, -1))) *
           inv_dx;
    DcDy = (dv.d3(Cs(0, 1) - Cs(0, -1)) + dv.d12(Cs(1, 1) + Cs(-1, 1) - Cs(1, -1) - Cs(-1, -1))) *
           inv_dx;
}

// Laplacian_AMR + Chemical_Potential_AMR (LBM_Subroutines.f90:94-112,316-333)
template <class DV, class CF>
__device__ __forceinline__ double chem_pot_f(DV& dv, const PhysD& ph, double inv_dx2, CF Cs) {
    const double D2C = dv.d6(Cs(-1, -1) + Cs(1, -1) + Cs(-1, 1) + Cs(1, 1) +
                             4.0 * (Cs(0, -1) + Cs(-1, 0) + Cs(1, 0) + Cs(0, 1)) - 20.0 * Cs(0, 0));
    const double c = Cs(0, 0);
    return ph.Beta4 * c * (c - 1.0) * (c - 0.5) - ph.kappa * D2C * inv_dx2;
}

// ---------------------------------------------------------------------------
// One-CTA bulk copies global -> shared (cp.async.bulk, completion counted in
// bytes on an mbarrier). Addresses 16-byte aligned, sizes multiples of 16.
// No cluster multicast: the source is always this GPU's own memory.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// Shared-memory load of data that stays unchanged while it is read (staged by
// a completed bulk copy), issued where it is written in the source: the
// collision then loads a population when it uses it instead of holding all
// of them in registers.
__device__ __forceinline__ double lds(const double* p) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)));
    return v;
}
// 4-byte asynchronous copy global -> shared (cp.async, no register staging);
// cp_async_wait_all waits for all of this thread's copies
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// generic-proxy accesses of shared memory before later bulk copies into it
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of bar; false if it ran out (the caller
// reports AMRLBM_ERR_TIMEOUT and carries on with whatever is in shared memory).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    for (int it = 0; it < 4000000; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}
