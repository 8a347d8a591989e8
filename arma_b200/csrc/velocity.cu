// Linear velocity-potential solver (placeholder until the FFT kernels land).
#include "internal.h"

namespace armab {

void launch_velocity_linear(Ctx*, const void*, const int*, int, const double*, double,
                            const double*, int, const int*, int, void*) {
	throw Error{ARMA_ENOTSUP, "linear velocity solver is not built yet"};
}

}  // namespace armab
