// Entry points of the reference's stl-bridge that belong to subsystems
// outside this engine: the spectrum engine (crates/stl-core/src/sht.rs) and the U-Net training
// (crates/stl-bridge/src/unet.rs).  The reference's native.py binds every
// name of its signature table when it loads the library, so each is
// exported here and fails with a message naming the subsystem.
#include <string>

#include "../../include/stl_b200.h"

namespace stl {
void set_error(const std::string& msg);
}

namespace {
int fail(const char* what) {
  stl::set_error(std::string(what) + " is not built in the B200 ScatCov engine library");
  return -1;
}
void* fail_ptr(const char* what) {
  fail(what);
  return nullptr;
}
}  // namespace

extern "C" {

void* stlp_spec_new(const char*) { return fail_ptr("the spectrum engine (stlp_spec_new)"); }
void stlp_spec_free(void*) {}
char* stlp_spec_info(void*) { return (char*)fail_ptr("the spectrum engine (stlp_spec_info)"); }
int stlp_spec_set_masks(void*, const double*, size_t) { return fail("the spectrum engine (stlp_spec_set_masks)"); }
int stlp_spec_forward(void*, const double*, size_t, uint64_t, uint64_t, uint64_t, double*) {
  return fail("the spectrum engine (stlp_spec_forward)");
}
int stlp_spec_vjp(void*, const double*, size_t, uint64_t, uint64_t, uint64_t, double*) {
  return fail("the spectrum engine (stlp_spec_vjp)");
}
void* stlp_unet_new(const char*) { return fail_ptr("the U-Net (stlp_unet_new)"); }
void stlp_unet_free(void*) {}
char* stlp_unet_info(void*) { return (char*)fail_ptr("the U-Net (stlp_unet_info)"); }
int stlp_unet_get_params(void*, float*) { return fail("the U-Net (stlp_unet_get_params)"); }
int stlp_unet_set_params(void*, const float*, size_t) { return fail("the U-Net (stlp_unet_set_params)"); }
int stlp_unet_get_grads(void*, float*) { return fail("the U-Net (stlp_unet_get_grads)"); }
int stlp_unet_zero_grad(void*) { return fail("the U-Net (stlp_unet_zero_grad)"); }
int stlp_unet_adam(void*, double) { return fail("the U-Net (stlp_unet_adam)"); }
int stlp_unet_set_cond(void*, const float*, size_t) { return fail("the U-Net (stlp_unet_set_cond)"); }
int stlp_unet_apply(void*, const double*, size_t, double*, double*, double*) {
  return fail("the U-Net (stlp_unet_apply)");
}
int stlp_train_set_masks(void*, const double*, size_t) { return fail("U-Net training (stlp_train_set_masks)"); }
int stlp_train_set_common(void*, const double*) { return fail("U-Net training (stlp_train_set_common)"); }
int stlp_train_set_field(void*, uint32_t, const double*, const double*, const double*, const double*, const double*,
                         const double*, size_t, double) {
  return fail("U-Net training (stlp_train_set_field)");
}
int stlp_train_bias(void*, uint32_t, const uint64_t*, const double*, size_t) {
  return fail("U-Net training (stlp_train_bias)");
}
int stlp_train_loss(void*, uint32_t, bool, double*) { return fail("U-Net training (stlp_train_loss)"); }
int stlp_train_step(void*, uint32_t, double, double*) { return fail("U-Net training (stlp_train_step)"); }
int stlp_train_live(void*, uint32_t, const uint64_t*, const double*, size_t, const uint64_t*, const double*, size_t,
                    bool, double, double*) {
  return fail("U-Net training (stlp_train_live)");
}
void* stlp_train_lbfgs(void*, const uint32_t*, size_t, const char*) {
  return fail_ptr("U-Net training (stlp_train_lbfgs)");
}
int stlp_train_set_joint(void*, const double*, const double*, uint32_t, uint32_t, const char*, double) {
  return fail("U-Net training (stlp_train_set_joint)");
}
int stlp_train_front(void*, const double*, size_t, bool, double*) { return fail("U-Net training (stlp_train_front)"); }

}  // extern "C"
