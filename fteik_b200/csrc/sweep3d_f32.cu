/*
 * sweep3d_f32.cu -- FP32 instantiation of the 3D solve (the product path):
 * FP32 travel times and plane-wave stencils, FP64 for the analytic source
 * corners, the near-source spherical stencil and the convergence residual.
 * The initialisation kernel is instantiated in slab_init_f32.cu.
 */
#include "row3d_impl.cuh"

namespace fk3tw {
cudaEvent_t *g_slab_events = nullptr;
}

extern "C" void fk3d_slabs_set_events(cudaEvent_t *ev3) { fk3tw::g_slab_events = ev3; }

extern "C" int fk3d_solve_slabs_f64(const fk_grid3d_t *grids, const fk_work3d_t *work, int nwork,
                                    const fk_slabs3d_t *plan, fk_result3d_t *results, double eps,
                                    int nsweep, double conv_tol, int max_pass, cudaStream_t stream);

extern "C" int fk3d_solve_slabs(int precision, const fk_grid3d_t *grids, const fk_work3d_t *work,
                                int nwork, const fk_slabs3d_t *plan, fk_result3d_t *results,
                                double eps, int nsweep, double conv_tol, int max_pass,
                                cudaStream_t stream)
{
    if (precision == 8)
        return fk3d_solve_slabs_f64(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                    max_pass, stream);
    if (precision != 4) return (int)cudaErrorInvalidValue;
    return fk3rw::launch_rows<float>(grids, work, nwork, plan, results, eps, nsweep, conv_tol,
                                     max_pass, stream);
}
