// kernels_af.cpp -- the reference's src/kernels.hpp implemented on
// libadaptflood.so: the file a maintainer compiles in place of the
// reference's src/kernels.cpp (src/kernels.hpp:8-37) to run its unmodified
// src/main.cpp loop on this library's CUDA kernels.
//
// Each function unwraps its views with .data() and calls the matching C ABI
// entry point (include/adaptflood.h) on the legacy default stream; every call
// returns after its kernels finish, as each reference function ends in
// Kokkos::fence().  The views of the reference are CudaUVMSpace
// (src/types.hpp:10-11): managed memory that both the device kernels and the
// host loops of src/main.cpp touch.  An error aborts the program, as Kokkos
// does in the reference.
#include <cstdio>
#include <cstdlib>

#include "adaptflood.h"
#include "kernels.hpp"

namespace {

void af_check(int rc, const char* what) {
  if (rc != AF_OK) {
    std::fprintf(stderr, "%s: %s %s\n", what, af_strerror(rc),
                 rc == AF_ECUDA ? af_last_cuda_error() : "");
    std::abort();
  }
}

}  // namespace

// src/kernels.cpp:6-19
void UpdateQs_GPU(RealView& Qx, RealView& Qy, RealView& Qxold, RealView& Qyold, int xsz,
                  int ysz, double dx) {
  af_check(af_update_qs(Qx.data(), Qy.data(), Qxold.data(), Qyold.data(), xsz, ysz, dx,
                        nullptr),
           "UpdateQs_GPU");
}

// src/kernels.cpp:22-146; Tstep is written before return.
void FloodplainQ_GPU(RealView& H, RealView& DEM, RealView& Qx, RealView& Qy, RealView& Qxold,
                     RealView& Qyold, int xsz, int ysz, double dx, double dy, double FPn,
                     double DepthThresh, double MaxHflow, double dhlin, double& Tstep,
                     double Qlimfact, double dA, double cfl, double g, double InitTstep,
                     double theta, double nodata) {
  af_check(af_floodplain_q(H.data(), DEM.data(), Qx.data(), Qy.data(), Qxold.data(),
                           Qyold.data(), xsz, ysz, dx, dy, FPn, DepthThresh, MaxHflow, dhlin,
                           &Tstep, Qlimfact, dA, cfl, g, InitTstep, theta, nodata, nullptr),
           "FloodplainQ_GPU");
}

// src/kernels.cpp:149-256
void BCs_GPU(RealView& Qx, RealView& Qy, RealView& H, RealView& DEM, int xsz, int ysz,
             double dx, double g, double dt, double nodata, bool west_free, bool east_free,
             bool north_free, bool south_free) {
  af_check(af_bcs(Qx.data(), Qy.data(), H.data(), DEM.data(), xsz, ysz, dx, g, dt, nodata,
                  west_free, east_free, north_free, south_free, nullptr),
           "BCs_GPU");
}

// src/kernels.cpp:259-277; the cell count bounds the indices.
void ApplyPointBCs_GPU(RealView& H, IntView& bc_idx, IntView& bc_type, RealView& bc_value,
                       int num_bcs, int ncols, double dx, double dA, double Tstep) {
  af_check(af_apply_point_bcs(H.data(), bc_idx.data(), bc_type.data(), bc_value.data(),
                              num_bcs, ncols, dx, dA, Tstep, (int)H.extent(0), nullptr),
           "ApplyPointBCs_GPU");
}

// src/kernels.cpp:280-290
void UpdateH_GPU(RealView& H, RealView& Qx, RealView& Qy, int xsz, int ysz, double dA,
                 double Tstep) {
  af_check(af_update_h(H.data(), Qx.data(), Qy.data(), xsz, ysz, dA, Tstep, nullptr),
           "UpdateH_GPU");
}

// src/kernels.cpp:293-351
void ComputeVelocity_GPU(RealView& Vx_out, RealView& Vy_out, RealView& H, RealView& DEM,
                         RealView& Qx, RealView& Qy, int xsz, int ysz, double dx,
                         double nodata) {
  af_check(af_compute_velocity(Vx_out.data(), Vy_out.data(), H.data(), DEM.data(), Qx.data(),
                               Qy.data(), xsz, ysz, dx, nodata, nullptr),
           "ComputeVelocity_GPU");
}

// src/kernels.cpp:354-367
void Rainfall_GPU(RealView& H, RealView& DEM, int xsz, int ysz, double rain_rate,
                  double Tstep, double nodata) {
  af_check(af_rainfall(H.data(), DEM.data(), xsz, ysz, rain_rate, Tstep, nodata, nullptr),
           "Rainfall_GPU");
}
