// Placeholder translation unit: registers no gradient kernels yet.
#include "dispatch.h"
#include "../../include/b200jk.h"
#include "plan.h"
namespace b200jk {
void register_grad_classes(DispatchTable&) {}
}
extern "C" {
int b200jk_direct_jk_geom_vjp(b200jk_plan*, const double*, int32_t, const double*, int32_t, int32_t,
                              double*, void*) { b200jk::set_error("not built"); return B200JK_UNSUPPORTED; }
int b200jk_int1e(b200jk_plan*, int32_t, double*, void*) { b200jk::set_error("not built"); return B200JK_UNSUPPORTED; }
int b200jk_int1e_grad(b200jk_plan*, const double*, const double*, double*, void*) { b200jk::set_error("not built"); return B200JK_UNSUPPORTED; }
}
