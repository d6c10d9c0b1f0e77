// Kernel launchers shared between the C-ABI layer and the kernel files.
#pragma once
#include <cuda_runtime.h>

#include "ctx.h"
#include "records.cuh"

namespace mochii {

int transport_blocks(const mochii_ctx* c);
cudaError_t launch_transport(mochii_ctx* c);
cudaError_t packet_order_alloc(mochii_ctx* c, long long cap);   // packet_order: keys, walk order, sort buffers
PacketRecords packet_records(mochii_ctx* c);
cudaError_t launch_transport_diffuse(mochii_ctx* c, double total, long long nd);
cudaError_t diffuse_build(mochii_ctx* c, double* total);
size_t diffuse_scan_bytes(long long nleaf);
// Records of diffuse packets ip0 .. ip0+n-1; with order, record i holds
// chunk packet order[i].
cudaError_t launch_diffuse_chunk(mochii_ctx* c, double total, long long ip0, long long n,
                                 const int* order = nullptr);
// diffuse_coherent_key of diffuse packets ip0 .. ip0+n-1 (Cartesian grid).
cudaError_t launch_diffuse_keys(mochii_ctx* c, double total, long long ip0, long long n, unsigned* key);
cudaError_t launch_rates(mochii_ctx* c);
cudaError_t peel_setup(mochii_ctx* c);   // par%ion_peel: observers, image plane, device images (peel.cpp)
cudaError_t peel_clear(mochii_ctx* c);   // zero the images before an imaging pass
cudaError_t launch_jt_export(mochii_ctx* c, double* dst);
cudaError_t launch_sobol(const QmcTables* t, int stream01, long long idx0, long long n, int nd, double* out,
                         cudaStream_t s);
cudaError_t launch_walk(mochii_ctx* c, const double* rays, long long nray, int max_steps, int* leaves, int* nsteps);
cudaError_t launch_philox(uint64_t seed, uint32_t stream, uint64_t packet, int n0, int n, double* out);
cudaError_t launch_records(mochii_ctx* c, long long ip0, long long n, double* out);
long long noalloc_max_records();
cudaError_t launch_records_from_buffer(mochii_ctx* c, long long n, double* host_out);
cudaError_t launch_records_noalloc(mochii_ctx* c, long long ip0, long long n, double* host_out);

int balance_blocks(const mochii_ctx* c);
cudaError_t launch_columns(mochii_ctx* c);
cudaError_t launch_metal_fractions(mochii_ctx* c, double* out);   // nleaf x nstages, registry order
cudaError_t launch_balance(mochii_ctx* c);
cudaError_t launch_thermal(mochii_ctx* c);
cudaError_t metal_ttable_build(mochii_ctx* c);   // the T table of the metal rate coefficients
cudaError_t nl_log_tables(const double* lamref, const double* Ssup, int ntab, double** out, cudaStream_t s);
cudaError_t thermal_work_alloc(mochii_ctx* c);
// batched nebulae: the one-launch lockstep thermal solve of several contexts
void* thermal_batch_create(mochii_ctx* const* cs, int n, cudaError_t* err);
void thermal_batch_destroy(void* tb);
cudaError_t thermal_batch_enqueue(void* tb, mochii_ctx* const* cs, cudaStream_t s);
cudaError_t thermal_batch_set_warm(void* tb, mochii_ctx* const* cs, const double* fac, double gate);
double mlp_step_factor(const mochii_mlp* m, double observed_ln = 0.0);
cudaError_t warm_error_launch(mochii_ctx* c);
// dust_temp_mod.f90: T_dust of every leaf into c->tdust; the IR spectrum of
// it (out_dev[0..239] = L_nu at the IR wavelengths, out_dev[240] = absorbed power)
cudaError_t dust_temp_launch(mochii_ctx* c);
cudaError_t dust_ir_launch(mochii_ctx* c, double* out_dev);
int mlp_batch_prepare(mochii_mlp* m, mochii_ctx* const* cs, int n, double* fac);
cudaError_t mlp_warm_start_enqueue(mochii_ctx* c, mochii_mlp* m, cudaStream_t s);

}  // namespace mochii
