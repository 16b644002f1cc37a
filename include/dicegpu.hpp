// dicegpu.hpp -- C++ host interface over the C ABI (header only).
//
// Mirrors the reference's boundary for the local-DIC hot path:
//   DICe::Schema(..., params)                  -> dicegpu::Schema(params)
//   Schema::set_ref_image(w, h, array)         -> set_ref_image(w, h, pixels)
//   Schema::set_def_image(w, h, array)         -> set_def_image(w, h, pixels)
//   Schema::execute_correlation()              -> execute_correlation()   (returns 0)
//   Schema::global_field_value(gid, field)     -> global_field_value(gid, column)
// (src/core/DICe_Schema.h:543-551, DICe_Schema.cpp:328-349, 1622).
// Errors from the library become dicegpu::Error exceptions on the C++ side;
// the C ABI underneath never throws.
#ifndef DICEGPU_HPP
#define DICEGPU_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "dicegpu.h"

namespace dicegpu {

class Error : public std::runtime_error {
 public:
  Error(const std::string& what, int code) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* what) {
  if (rc != DICEGPU_OK) throw Error(std::string(what) + " failed with code " + std::to_string(rc), rc);
}

inline dicegpu_params default_params() {
  dicegpu_params p;
  check(dicegpu_default_params(&p), "dicegpu_default_params");
  return p;
}

class Schema {
 public:
  explicit Schema(const dicegpu_params& params) : params_(params) {
    check(dicegpu_create(&params_, &ctx_), "dicegpu_create");
  }
  ~Schema() {
    if (ctx_) dicegpu_destroy(ctx_);
  }
  Schema(const Schema&) = delete;
  Schema& operator=(const Schema&) = delete;

  const dicegpu_params& params() const { return params_; }
  void set_params(const dicegpu_params& p) {
    check(dicegpu_set_params(ctx_, &p), "dicegpu_set_params");
    params_ = p;
  }
  void set_stream(void* stream) { check(dicegpu_set_stream(ctx_, stream), "dicegpu_set_stream"); }

  void set_ref_image(int w, int h, const float* pixels, bool on_device = false) {
    check(dicegpu_set_ref_image(ctx_, w, h, pixels, on_device ? 1 : 0), "dicegpu_set_ref_image");
  }
  void set_def_image(int w, int h, const float* pixels, bool on_device = false) {
    check(dicegpu_set_def_image(ctx_, w, h, pixels, on_device ? 1 : 0), "dicegpu_set_def_image");
  }

  // Square subsets centred on (cx[i], cy[i]) with zero initial motion.
  void set_subsets(const std::vector<double>& cx, const std::vector<double>& cy) {
    if (cx.size() != cy.size() || cx.empty()) throw Error("set_subsets: bad coordinates", DICEGPU_ERR_ARG);
    fields_.assign(cx.size() * DICEGPU_FIELD_STRIDE, 0.0);
    for (size_t i = 0; i < cx.size(); ++i) {
      fields_[i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X] = cx[i];
      fields_[i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y] = cy[i];
      if (params_.shape_function == DICEGPU_QUADRATIC_SF) {
        fields_[i * DICEGPU_FIELD_STRIDE + DICEGPU_F_QUAD_A] = 1.0;
        fields_[i * DICEGPU_FIELD_STRIDE + DICEGPU_F_QUAD_A + 7] = 1.0;
      }
    }
    set_fields(fields_);
  }
  void set_fields(const std::vector<double>& f) {
    if (f.empty() || f.size() % DICEGPU_FIELD_STRIDE) throw Error("set_fields: bad size", DICEGPU_ERR_ARG);
    fields_ = f;
    n_ = (int)(f.size() / DICEGPU_FIELD_STRIDE);
    check(dicegpu_set_subsets(ctx_, n_, fields_.data()), "dicegpu_set_subsets");
    fresh_ = true;
  }

  // Conformal subsets (Conformal_Area_Def shapes) and obstructing subsets
  // (obstructing_subset_ids_ in CSR form: offsets[n + 1], ids).
  void set_subset_shapes(const std::vector<dicegpu_shape>& shapes, const std::vector<int32_t>& vx,
                         const std::vector<int32_t>& vy) {
    check(dicegpu_set_subset_shapes(ctx_, (int)shapes.size(), shapes.data(), vx.empty() ? nullptr : vx.data(),
                                    vy.empty() ? nullptr : vy.data()),
          "dicegpu_set_subset_shapes");
  }
  void set_blocking(const std::vector<int32_t>& offsets, const std::vector<int32_t>& ids) {
    check(dicegpu_set_blocking(ctx_, offsets.empty() ? nullptr : offsets.data(), ids.empty() ? nullptr : ids.data()),
          "dicegpu_set_blocking");
  }
  // NEIGHBOR_ID per subset for the neighbour initializers.
  void set_neighbors(const std::vector<int32_t>& ids) {
    if ((int)ids.size() != n_) throw Error("set_neighbors: one id per subset", DICEGPU_ERR_ARG);
    check(dicegpu_set_neighbors(ctx_, ids.data()), "dicegpu_set_neighbors");
  }
  // set_ref_image(prev_img()) of an incremental sequence: the current
  // deformed image becomes the reference on the device.
  void set_ref_from_def() { check(dicegpu_set_ref_from_def(ctx_), "dicegpu_set_ref_from_def"); }

  // One frame over every subset; returns 0 as Schema::execute_correlation does.
  int execute_correlation() {
    check(dicegpu_execute_correlation(ctx_), "dicegpu_execute_correlation");
    fresh_ = false;
    return 0;
  }

  int num_subsets() const { return n_; }
  const std::vector<double>& fields() {
    if (!fresh_) {
      check(dicegpu_get_fields(ctx_, fields_.data()), "dicegpu_get_fields");
      fresh_ = true;
    }
    return fields_;
  }
  double global_field_value(int subset, int column) {
    if (subset < 0 || subset >= n_ || column < 0 || column >= DICEGPU_FIELD_STRIDE)
      throw Error("global_field_value: index out of range", DICEGPU_ERR_ARG);
    return fields()[(size_t)subset * DICEGPU_FIELD_STRIDE + column];
  }

  dicegpu_ctx* handle() { return ctx_; }

 private:
  dicegpu_params params_;
  dicegpu_ctx* ctx_ = nullptr;
  std::vector<double> fields_;
  int n_ = 0;
  bool fresh_ = false;
};

}  // namespace dicegpu

#endif  // DICEGPU_HPP
