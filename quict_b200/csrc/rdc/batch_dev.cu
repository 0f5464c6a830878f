// The persistent batch kernel as relocatable device code.  quict_b200/build.py
// compiles this file to an sm_100a cubin (nvcc -rdc -cubin) and embeds it in
// libqsim.so; at run time it is linked (nvJitLink, csrc/jit.cu) with the
// register-stage functions generated for a plan and their dispatcher
// qs_batch_jit, so that those stages run as straight-line code inside the one
// persistent launch.  Stages without a generated function run the generic
// register body, as in the kernel of batch.cu.
#include "../batch.cuh"

extern "C" __global__ void __launch_bounds__(256, 1)
qs_batch_linked_c64(const unsigned char* __restrict__ blob, float2* __restrict__ states,
                    const float2* __restrict__ mats, double* __restrict__ parts, double* __restrict__ energies,
                    double* __restrict__ grads, unsigned long long* __restrict__ ctrl, uint64_t timeout_ns) {
    qs::batch_loop<float2, 5, true>(blob, states, mats, parts, energies, grads, ctrl, timeout_ns);
}

extern "C" __global__ void __launch_bounds__(256, 1)
qs_batch_linked_c128(const unsigned char* __restrict__ blob, double2* __restrict__ states,
                     const double2* __restrict__ mats, double* __restrict__ parts, double* __restrict__ energies,
                     double* __restrict__ grads, unsigned long long* __restrict__ ctrl, uint64_t timeout_ns) {
    qs::batch_loop<double2, 4, true>(blob, states, mats, parts, energies, grads, ctrl, timeout_ns);
}
