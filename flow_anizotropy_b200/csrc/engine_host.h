// Host-side pieces shared by the engine translation units (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>

#include "../../include/lbm.h"
#include "engine3d.cuh"

struct lbm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sms = 0;
    std::string err;
    // test knobs of the bulk-staged odd step (lbm_debug_bulk_wait): wait
    // limit in ns (0: the kernels' own), and a producer that issues nothing
    unsigned long long test_wait_ns = 0;
    int test_starve = 0;
};

int lbm_fail_cuda(lbm_ctx *ctx, cudaError_t e, const char *what, int line);
int lbm_fail_input(lbm_ctx *ctx, const std::string &msg);
// The step-kernel variant LBM_VARIANT_DEFAULT stands for.
int lbm_default_variant(int prec);
int lbm_default_batch_variant(int prec);
// Deferred flux reduction (StepArgs::defer) for this precision, and the
// doubles of a solve's partials buffer with it.
bool lbm_defers(int prec);
long long lbm_partial_doubles(int prec, int ntiles);
bool lbm_is_device_ptr(const void *p);
std::string &lbm_last_error_global();

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return lbm_fail_cuda(ctx, e_, #call, __LINE__); \
    } while (0)

// Stream-ordered device allocation released when the owner goes out of scope.
struct DevMem {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    explicit DevMem(cudaStream_t st) : s(st) {}
    DevMem(const DevMem &) = delete;
    DevMem &operator=(const DevMem &) = delete;
    DevMem(DevMem &&o) noexcept : p(o.p), s(o.s) { o.p = nullptr; }
    DevMem &operator=(DevMem &&o) noexcept
    {
        if (this != &o) { release(); p = o.p; s = o.s; o.p = nullptr; }
        return *this;
    }
    ~DevMem() { release(); }
    cudaError_t alloc(size_t n)
    {
        release();
        return cudaMallocAsync(&p, n ? n : 16, s);
    }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
    }
};

int lbm_upload_mask(lbm_ctx *ctx, const uint8_t *solid, int nx, long long rows, DevMem &mask,
                    long long &npore);
int lbm_check_params3d(lbm_ctx *ctx, const lbm_params3d &p);
long long lbm_plane_elems(long long nn);
long long lbm_lattice_bytes3d(long long nn, int prec);
// Lattice bytes of one direction of a filled solve record (any storage form).
long long lbm_lattice_bytes(const lbm::Solve3 &S);
void lbm_fill_solve3(lbm::Solve3 &S, int nx, int ny, int nz, const double F[3], const lbm_params3d &p, int npt);
void lbm_init_state3(lbm::State3 &st, const lbm::Ctl3 &c);
int lbm_pick_npt(const lbm_params3d &p);
// Pore-rank tables of a structure (wpre, fnode of S; nfluid, plane, ntiles for npt).
int lbm_build_pores(lbm_ctx *ctx, lbm::Solve3 &S, int npt, DevMem &wpre, DevMem &fnode, DevMem &meta,
                    DevMem &meta2);
int lbm_effective_variant(int prec, int variant, bool have_meta);
// Does the variant step a structure's directions in one work item (grouped work list)?
bool lbm_grouped_variant(int prec, int variant);
// ... and do all of its launches (the grouped pull form)?
bool lbm_grouped_all(int prec, int variant);
void lbm_attach_lattice(lbm::Solve3 &S, void *p);
void lbm_copy_pores(lbm::Solve3 &dst, const lbm::Solve3 &src);
cudaError_t lbm_launch_step(int prec, int variant, bool w1, bool odd, dim3 grid, cudaStream_t s, const lbm::StepArgs &a);
int lbm_max_blocks(int prec, int variant, bool odd);
cudaError_t lbm_init_lattice(int prec, const lbm::Solve3 &S, cudaStream_t s);
cudaError_t lbm_canon(int prec, const lbm::Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
