// tc_complex.cu — split-BF16 tcgen05 tensor-core kernels (signal, J·v, Jᴴ·v).
#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {

bool launch_signal_cartesian_tc(const CompasContext&, const float*, int64_t, int, const cfloat*, const cfloat*, int,
                                const CartesianGeom&, cfloat*) {
    return false;
}

bool launch_jacobian_tc(const CompasContext&, const float*, int64_t, int, const cfloat*, const cfloat*, const cfloat*,
                        const cfloat*, int, const cfloat*, const CartesianGeom&, cfloat*) {
    return false;
}

bool launch_jacobian_hermitian_tc(const CompasContext&, const float*, int64_t, int, const cfloat*, const cfloat*,
                                  const cfloat*, const cfloat*, int, const cfloat*, const CartesianGeom&, cfloat*) {
    return false;
}

}  // namespace compas
