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
// extract, poisson_phi: odd-extended complex arrays and the dead Jacobi
// iteration) have no counterpart: the library's solve never forms the
// odd-extended array.  A caller that used them directly calls fast_Poisson.
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
