/*
 * sweep3d_f32.cu -- FP32 instantiation of the 3D solve (the product path):
 * FP32 travel times and plane-wave stencils, FP64 for the analytic source
 * corners, the near-source spherical stencil and the convergence residual.
 */
#include "sweep3d_impl.cuh"
#include "tile3d_impl.cuh"
#include "row3d_impl.cuh"

namespace fk3tw {
cudaEvent_t *g_tile_events = nullptr;
}

extern "C" void fk3d_tiles_set_events(cudaEvent_t *ev3) { fk3tw::g_tile_events = ev3; }

extern "C" int fk3d_solve_f64(const fk_grid3d_t *grids, const fk_work3d_t *work,
                              const int *groups, int ngroups, int S, fk_result3d_t *results,
                              int nwork, int max_nx, int max_nz, double eps, int nsweep,
                              double conv_tol, int max_pass, cudaStream_t stream);
extern "C" int fk3d_prepare_f64(int max_nx, int max_nz, int S);
extern "C" int fk3d_pick_s_f64(int max_nx, int max_nz, int nwork, int nsm);

extern "C" int fk3d_solve(int precision, const fk_grid3d_t *grids, const fk_work3d_t *work,
                          const int *groups, int ngroups, int S, fk_result3d_t *results,
                          int nwork, int max_nx, int max_nz, double eps, int nsweep,
                          double conv_tol, int max_pass, cudaStream_t stream)
{
    if (S != 1 && S != 2) return (int)cudaErrorInvalidValue;
    if (precision == 8)
        return fk3d_solve_f64(grids, work, groups, ngroups, S, results, nwork, max_nx, max_nz, eps,
                              nsweep, conv_tol, max_pass, stream);
    if (precision != 4) return (int)cudaErrorInvalidValue;
    return fk3::launch_solve<float>(grids, work, groups, ngroups, S, results, nwork, max_nx,
                                    max_nz, eps, nsweep, conv_tol, max_pass, stream);
}

extern "C" int fk3d_prepare(int precision, int max_nx, int max_nz, int S)
{
    if (precision == 8) return fk3d_prepare_f64(max_nx, max_nz, S);
    return fk3::prepare_solve<float>(max_nx, max_nz, S);
}

extern "C" int fk3d_pick_s(int precision, int max_nx, int max_nz, int nwork)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (precision == 8) return fk3d_pick_s_f64(max_nx, max_nz, nwork, nsm);
    return fk3::pick_s<float>(max_nx, max_nz, nwork, nsm);
}

extern "C" size_t fk3d_smem_bytes(int precision, int max_nx, int max_nz)
{
    const int nt = ((max_nx + 31) / 32) * 32;
    return precision == 8 ? fk3::smem_need<double, 1>(nt, max_nz) : fk3::smem_need<float, 1>(nt, max_nz);
}

extern "C" int fk3d_solve_tiles_f64(const fk_grid3d_t *grids, const fk_work3d_t *work, int nwork,
                                    const fk_tiles3d_t *plan, fk_result3d_t *results, double eps,
                                    int nsweep, double conv_tol, int max_pass, cudaStream_t stream);

extern "C" int fk3d_solve_tiles(int precision, const fk_grid3d_t *grids, const fk_work3d_t *work,
                                int nwork, const fk_tiles3d_t *plan, fk_result3d_t *results,
                                double eps, int nsweep, double conv_tol, int max_pass,
                                cudaStream_t stream)
{
    if (precision == 8)
        return fk3d_solve_tiles_f64(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                    max_pass, stream);
    if (precision != 4) return (int)cudaErrorInvalidValue;
    if (plan->kind == FK_PLAN_ROWS)
        return fk3rw::launch_rows<float>(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                         max_pass, stream);
    return fk3tw::launch_tiles<float>(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                      max_pass, stream);
}
