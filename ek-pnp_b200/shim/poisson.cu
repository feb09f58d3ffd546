// poisson.cu (drop-in) -- fast_Poisson and efield of the reference's LBM.h
// (LBM.h:164-169) over libekpnp's C ABI; the companion of this folder's
// LBM.cu, which holds the shared state (see its header for the build line).
//
// fast_Poisson (poisson.cu:180-208 of the reference) writes psi, Ex and Ey to
// the globals phi_gpu, Ex_gpu, Ey_gpu, as the reference's does.  Called right
// after stream_collide_save it only completes that loop body: ek_step already
// ran the solve of the step, and the fields go to the caller's buffers on the
// steps whose results main.cu reads.  Called on its own it solves for the
// charges it is given, with no device allocation (the reference allocates and
// frees four buffers per call, poisson.cu:182-207).
//
// The reference's helpers of its cuFFT pipeline (extension, derivative,
// extract: odd-extended complex arrays) have no counterpart: the library's
// solve never forms the odd-extended array.  A caller that used them
// directly calls fast_Poisson.  poisson_phi, the reference's iterative
// solver (poisson.cu:35-130, not called by main.cu), runs the library's
// grid relaxation (ek_poisson_jacobi).
#ifndef EKPNP_SHIM_POISSON_CU
#define EKPNP_SHIM_POISSON_CU

#include "LBM.cu"

__host__ void fast_Poisson(double *charge_d, double *T_d, double *kx_, double *ky_, cufftHandle plan_) {
    (void)kx_, (void)ky_, (void)plan_;
    using namespace ekshim;
    State &s = st();
    if (s.step_open) {
        s.step_open = false;
        if (s.write_back) write_back_now();
        return;
    }
    checkCudaErrors(cudaDeviceSynchronize());  // the caller's charges are complete
    check(ek_set_fields_device(ctx(), nullptr, nullptr, nullptr, charge_d, T_d, nullptr, nullptr, nullptr),
          "ek_set_fields_device");
    check(ek_poisson(ctx()), "ek_poisson");
    check(ek_get_fields_device(ctx(), nullptr, nullptr, nullptr, nullptr, nullptr, phi_gpu, Ex_gpu, Ey_gpu),
          "ek_get_fields_device");
    check(ek_sync(ctx()), "ek_sync");
}

// c+ = rho_e / f_charge, c- = 0: the library's right-hand side
// -f_charge (c+ - c-) / eps is then the reference's -rho_e / eps.
__global__ void ekshim_charge_to_cp(const double *rho_e, double *cp, double *cn, double inv_f, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        cp[i] = rho_e[i] * inv_f;
        cn[i] = 0.0;
    }
}

// poisson_phi (poisson.cu:35-73): psi for the net charge density in
// charge_d by grid relaxation from the potential in phi_d, walls at
// voltage / voltage2, until the largest change of a sweep is below 1e-9 or
// 1e6 sweeps, then psi into phi_d.  The library's sweeps read one buffer and
// write another, so unlike the reference's in-place update the result does
// not depend on the block schedule; the change is measured every 100 sweeps
// instead of after every one.
__host__ void poisson_phi(double *charge_d, double *phi_d) {
    using namespace ekshim;
    const int n = (int)(NX * NY);
    double *cp = nullptr, *cn = nullptr;
    checkCudaErrors(cudaMalloc(&cp, mem_size_scalar));
    checkCudaErrors(cudaMalloc(&cn, mem_size_scalar));
    ekshim_charge_to_cp<<<(n + 255) / 256, 256>>>(charge_d, cp, cn, 1.0 / from_symbol(convertCtoCharge), n);
    checkCudaErrors(cudaGetLastError());
    checkCudaErrors(cudaDeviceSynchronize());
    check(ek_set_fields_device(ctx(), nullptr, nullptr, nullptr, cp, cn, phi_d, nullptr, nullptr),
          "ek_set_fields_device");
    int32_t sweeps = 0;
    double change = 0.0;
    const int32_t max_sweeps = 1000000;
    check(ek_poisson_jacobi(ctx(), max_sweeps, 1.0e-9, 1.0, 100, &sweeps, &change), "ek_poisson_jacobi");
    check(ek_get_fields_device(ctx(), nullptr, nullptr, nullptr, nullptr, nullptr, phi_d, nullptr, nullptr),
          "ek_get_fields_device");
    check(ek_sync(ctx()), "ek_sync");
    checkCudaErrors(cudaFree(cp));
    checkCudaErrors(cudaFree(cn));
    if (!(change < 1.0e-9)) {
        printf("Poisson solver did not converge!\n");
        printf("Residual = %g\n", change);
    }
}

// E = -grad psi with the reference's stencil (gpu_efield + gpu_bc,
// poisson.cu:132-174) for the potential in phi_d.
__host__ void efield(double *phi_d, double *Ex_d, double *Ey_d) {
    using namespace ekshim;
    checkCudaErrors(cudaDeviceSynchronize());
    check(ek_set_fields_device(ctx(), nullptr, nullptr, nullptr, nullptr, nullptr, phi_d, nullptr, nullptr),
          "ek_set_fields_device");
    check(ek_get_fields_device(ctx(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, Ex_d, Ey_d),
          "ek_get_fields_device");
    check(ek_sync(ctx()), "ek_sync");
}

#endif  // EKPNP_SHIM_POISSON_CU
