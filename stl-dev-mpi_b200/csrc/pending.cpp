// Entry points whose engine is added next (disc patches).
#include <string>

#include "../../include/stl_b200.h"

namespace stl {
void set_error(const std::string& msg);
}

namespace {
int fail(const char* what) {
  stl::set_error(std::string(what) + " is not built in this library yet");
  return -1;
}
}  // namespace

extern "C" {
StlpPatchHandle* stlp_patch_new(const char*) { fail("stlp_patch_new"); return nullptr; }
void stlp_patch_free(StlpPatchHandle*) {}
char* stlp_patch_info(StlpPatchHandle*) { fail("stlp_patch_info"); return nullptr; }
int stlp_pixel_vectors(size_t, const int64_t*, size_t, double*) { return fail("stlp_pixel_vectors"); }
int stlp_patch_select(StlpPatchHandle*, const double*, size_t, double, double, size_t*) { return fail("stlp_patch_select"); }
int stlp_patch_ids(StlpPatchHandle*, size_t, int64_t*) { return fail("stlp_patch_ids"); }
int stlp_patch_core_pixels(StlpPatchHandle*, size_t*) { return fail("stlp_patch_core_pixels"); }
int stlp_patch_forward(StlpPatchHandle*, const double*, size_t, uint64_t, bool, double*, double*) { return fail("stlp_patch_forward"); }
int stlp_patch_vjp(StlpPatchHandle*, const double*, size_t, uint64_t, double*) { return fail("stlp_patch_vjp"); }
int stlp_patch_forward_device(StlpPatchHandle*, uint64_t, size_t, uint64_t, bool, double*, double*) { return fail("stlp_patch_forward_device"); }
int stlp_patch_vjp_device(StlpPatchHandle*, const double*, size_t, uint64_t, uint64_t) { return fail("stlp_patch_vjp_device"); }
}
