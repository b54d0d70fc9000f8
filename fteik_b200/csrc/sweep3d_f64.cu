/*
 * sweep3d_f64.cu -- FP64 instantiation of the 3D solve.  Compiled without
 * multiply-add contraction so that it reproduces the FP64 CPU algorithm's
 * rounding; used to check the kernels' schedule, masks and stencils exactly
 * and offered as a full-precision mode.
 */
#include "row3d_impl.cuh"

extern "C" int fk3d_solve_slabs_f64(const fk_grid3d_t *grids, const fk_work3d_t *work, int nwork,
                                    const fk_slabs3d_t *plan, fk_result3d_t *results, double eps,
                                    int nsweep, double conv_tol, int max_pass, cudaStream_t stream)
{
    return fk3rw::launch_rows<double>(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                      max_pass, stream);
}
