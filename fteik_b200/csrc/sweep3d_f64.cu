/*
 * sweep3d_f64.cu -- FP64 instantiation of the 3D solve.  Compiled without
 * multiply-add contraction so that it reproduces the FP64 CPU algorithm's
 * rounding; used to check the kernels' schedule, masks and stencils exactly
 * and offered as a full-precision mode.
 */
#include "sweep3d_impl.cuh"
#include "tile3d_impl.cuh"
#include "row3d_impl.cuh"

extern "C" int fk3d_solve_f64(const fk_grid3d_t *grids, const fk_work3d_t *work,
                              const int *groups, int ngroups, int S, fk_result3d_t *results,
                              int nwork, int max_nx, int max_nz, double eps, int nsweep,
                              double conv_tol, int max_pass, cudaStream_t stream)
{
    return fk3::launch_solve<double>(grids, work, groups, ngroups, S, results, nwork, max_nx,
                                     max_nz, eps, nsweep, conv_tol, max_pass, stream);
}

extern "C" int fk3d_prepare_f64(int max_nx, int max_nz, int S)
{
    return fk3::prepare_solve<double>(max_nx, max_nz, S);
}

extern "C" int fk3d_pick_s_f64(int max_nx, int max_nz, int nwork, int nsm)
{
    return fk3::pick_s<double>(max_nx, max_nz, nwork, nsm);
}

extern "C" int fk3d_solve_tiles_f64(const fk_grid3d_t *grids, const fk_work3d_t *work, int nwork,
                                    const fk_tiles3d_t *plan, fk_result3d_t *results, double eps,
                                    int nsweep, double conv_tol, int max_pass, cudaStream_t stream)
{
    if (plan->kind == FK_PLAN_ROWS)
        return fk3rw::launch_rows<double>(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                          max_pass, stream);
    return fk3tw::launch_tiles<double>(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                       max_pass, stream);
}
