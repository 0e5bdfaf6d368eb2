// vd_host.h -- host-side services of vd_abi.cu used by the batch layer (vd_batch.cu).
#pragma once
#include <cstdint>
#include <vector>
#include "../../include/vidyut_b200.h"
#include "vd_kernels.cuh"

namespace vd_host {

// Records msg as this thread's vd_last_error() and returns code.
int set_error(int code, const char* msg);
// Uploads the loaded mechanism to the current device if needed (VD_OK or a status).
int ensure_mech(cudaStream_t st);
// The species count, electron index, mobility kinds and charges of the loaded
// mechanism and its generation (incremented by every vd_mech_init); VD_ERR_MECH
// when none is loaded.
struct MechInfo {
    int ns, e_id, generation;
    int mob_kind[VD_MAX_SPECIES + 1];
    int charge[VD_MAX_SPECIES];
};
int mech_info(MechInfo* out);
// Molecular weight [g/mol] of species s of the loaded mechanism (0 when none).
double species_mw(int s);
// Validation of a box + parameter block as vd_explicit_update_all does it.
int check_update_params(const vd_box* bx, const vd_params* p, const MechInfo& m);
// Fills the per-box transport record (everything but the array views and ntile).
void fill_transport_args(vd::TransportArgs& a, const vd_box* bx, const vd_params* p, const MechInfo& m);
int stencil_halo(int hyp_order);
// Per-call scratch from the library's stream-ordered pool on the current device
// (set up by ensure_mech); release it with cudaFreeAsync on the same stream.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st);
// Ids of the resident cases of a batch that met a NaN or infinity (vd_batch.cu);
// waits for the batch's queued work.  Those cases take no further steps.
int batch_failed_cases(vd_batch* b, std::vector<int>* ids);

}  // namespace vd_host
