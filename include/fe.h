/* fe.h — the C ABI of the B200 (sm_100a) backend for Field Engine laws.
 *
 * Plain pointers and sizes only. Every call returns an int status (FE_OK = 0, else an FE_E* code) and leaves a message
 * for fe_last_error() on the calling thread; no call throws or aborts. Host pointers passed in are read or written only
 * during the call. Device pointers are CUDA device addresses on the current device; `stream` is a cudaStream_t (NULL =
 * the legacy default stream).
 *
 * Each function names the reference interface it replaces (file:line in NotTruecCoder/online-physics-cuda).
 */
#ifndef FE_H
#define FE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FE_OK 0
#define FE_EINVAL 1    /* bad argument (sizes, ids, null pointers) */
#define FE_ENODEV 2    /* no usable sm_100 device / driver */
#define FE_ECUDA 3     /* a CUDA runtime, driver or NVRTC call failed */
#define FE_ELAW 4      /* the law does not compile (parse or validation errors) */
#define FE_EUNSUP 5    /* the law uses an op this backend does not run */
#define FE_EKERNEL 6   /* a kernel reported an error word (for example a bounded wait that gave up) */

/* ---- library ------------------------------------------------------------------------------------------------- */

/* ABI version (major * 1000 + minor). */
int fe_version(void);
/* The message of the last failing call on this thread ("" if none). */
const char* fe_last_error(void);
/* Whether an sm_100 device is usable; FE_ENODEV with the reason otherwise. Replaces CudaSolver::unavailable
 * (src/field/cuda/CudaSolver.hpp:30-32). */
int fe_device_check(void);

/* ---- contract record ---------------------------------------------------------------------------------------------
 * What one fused pass records per checked field (the reference keeps these in its record words R, filled by k_rows /
 * k_planes / k_range / k_bounds: src/field/cuda/CudaCodegen.cpp:182-250, judged in CudaSolver.cpp:530-571). */
typedef struct fe_check {
    double before;      /* sum of the field before the term (FP64, fixed order) */
    double before_abs;  /* sum of |field| before the term */
    double after;       /* sum after the term */
    double after_abs;
    uint32_t out_of_range;
    uint32_t not_finite;
    uint32_t first_bad; /* ~(linear index of the first bad cell); 0 if none */
    uint32_t lo_inv;    /* ~key of the least value after the pass (fe_key_to_float(~lo_inv)) */
    uint32_t hi_key;    /* key of the largest value (fe_key_to_float(hi_key)); 0 = no finite value seen */
    uint32_t changed;   /* any cell moved */
    uint32_t pad[2];
} fe_check;

float fe_key_to_float(uint32_t key);

/* ---- the hand-written 7-point heat step --------------------------------------------------------------------------
 * d T = diffuse(k, T) with one k: next = T + ((max(k,0) * acc) / (h*h)) * dt, acc the sum of (neighbour - T) over the
 * faces inside the lattice in the order -x,+x,-y,+y,-z,+z. The bit-identity witness for the generated step; replaces the
 * reference's hand-written `heat` kernel (bench/stencil_bench.cpp:46-65), in the law's operation order.
 *
 * T_dev and out_dev: nx*ny*nz floats (x fastest), distinct buffers. variant: 0..3 picks the TMA tile (see fe_heat7_rows),
 * -1 the plain-load kernel (any nx). zchunk: z-planes a CTA marches (>= 1). With `check` non-zero the pass fills the
 * fe_check at the start of `workspace` (FE_HEAT7_BEFORE / FE_HEAT7_AFTER say which totals); workspace holds
 * fe_heat7_workspace_bytes(...) bytes and must be reset by fe_check_reset before the pass. */
#define FE_HEAT7_BEFORE 1
#define FE_HEAT7_AFTER 2
size_t fe_heat7_workspace_bytes(int nx, int ny, int nz, int variant, int zchunk);
int fe_heat7_rows(int variant);
int fe_heat7_step(const float* T_dev, float* out_dev, int nx, int ny, int nz, float k, float h, float dt, float lo, float hi,
    int variant, int zchunk, int check, void* workspace, void* stream);
/* Sets a workspace's fe_check and error word to their empty state (all zero bytes) on `stream`, asynchronously. */
int fe_check_reset(void* workspace, void* stream);
/* Copies the fe_check at the start of `workspace` to the host (synchronises `stream`); also reports a kernel error word
 * as FE_EKERNEL. */
int fe_check_read(const void* workspace, fe_check* out, void* stream);

/* A device-to-device copy of n floats (n a multiple of 4, 16-byte aligned): the bandwidth roof for the roofline. */
int fe_copy_f32(const float* src_dev, float* dst_dev, size_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FE_H */
