// dicegpu_autograd.cpp -- the subset objective as a libtorch autograd
// Function over the C ABI of libdicegpu.so.
//
// SubsetObjective(params, def_image) -> per-subset objective (gamma, or the
// Gauss-Newton least-squares objective) of a dicegpu context's subsets at
// the given shape-function parameters on the given deformed image.  backward
// runs dicegpu_adjoint with the incoming gradient as the per-subset seed and
// returns the derivatives with respect to the parameters and to every pixel
// of the deformed image.  The reference has no derivative code; this is the
// entry a gradient-based fit of a global displacement model (for instance a
// B-spline control grid) uses through torch.
#include <torch/extension.h>
#include <ATen/cuda/CUDAContext.h>

#include "dicegpu.h"

namespace {

using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

void check(int rc, const char* what) {
  TORCH_CHECK(rc == DICEGPU_OK, "dicegpu ", what, " failed with code ", rc);
}

dicegpu_ctx* as_ctx(int64_t handle) { return reinterpret_cast<dicegpu_ctx*>(handle); }

// The context's field rows with the shape-function columns replaced by
// `params` (n x 6 affine in slot order u, v, theta, ex, ey, gxy; n x 12
// quadratic A..L).
torch::Tensor rows_for(dicegpu_ctx* ctx, const torch::Tensor& params, bool quadratic) {
  int n = 0;
  check(dicegpu_num_subsets(ctx, &n), "num_subsets");
  TORCH_CHECK(params.dim() == 2 && params.size(0) == n, "params must be n_subsets x P");
  TORCH_CHECK(params.size(1) == (quadratic ? 12 : 6), "params must have 6 (affine) or 12 (quadratic) columns");
  double* rows_ptr = nullptr;
  check(dicegpu_fields_device_ptr(ctx, &rows_ptr), "fields_device_ptr");
  auto opts = torch::TensorOptions().dtype(torch::kFloat64).device(params.device());
  torch::Tensor rows = torch::from_blob(rows_ptr, {n, DICEGPU_FIELD_STRIDE}, opts).clone();
  rows.narrow(1, quadratic ? DICEGPU_F_QUAD_A : DICEGPU_F_DISP_X, params.size(1))
      .copy_(params.to(torch::kFloat64));
  return rows;
}

void upload(dicegpu_ctx* ctx, const torch::Tensor& def_image) {
  TORCH_CHECK(def_image.is_cuda() && def_image.dtype() == torch::kFloat32 && def_image.dim() == 2,
              "def_image must be a 2-D float32 CUDA tensor");
  check(dicegpu_set_stream(ctx, at::cuda::getCurrentCUDAStream().stream()), "set_stream");
  torch::Tensor img = def_image.contiguous();
  check(dicegpu_set_def_image(ctx, (int)img.size(1), (int)img.size(0), img.data_ptr<float>(), 1),
        "set_def_image");
}

class SubsetObjective : public torch::autograd::Function<SubsetObjective> {
 public:
  static torch::Tensor forward(AutogradContext* actx, torch::Tensor params, torch::Tensor def_image,
                               int64_t handle, int64_t objective, bool quadratic) {
    dicegpu_ctx* ctx = as_ctx(handle);
    TORCH_CHECK(params.is_cuda(), "params must be a CUDA tensor");
    upload(ctx, def_image);
    torch::Tensor rows = rows_for(ctx, params, quadratic);
    torch::Tensor value = torch::empty({params.size(0)}, rows.options());
    check(dicegpu_adjoint(ctx, rows.data_ptr<double>(), nullptr, (int)objective, 0,
                          value.data_ptr<double>(), nullptr, nullptr),
          "adjoint (forward)");
    actx->save_for_backward({params, def_image});
    actx->saved_data["handle"] = handle;
    actx->saved_data["objective"] = objective;
    actx->saved_data["quadratic"] = quadratic;
    return value.to(params.dtype());
  }

  static tensor_list backward(AutogradContext* actx, tensor_list grad_out) {
    auto saved = actx->get_saved_variables();
    torch::Tensor params = saved[0], def_image = saved[1];
    dicegpu_ctx* ctx = as_ctx(actx->saved_data["handle"].toInt());
    const int64_t objective = actx->saved_data["objective"].toInt();
    const bool quadratic = actx->saved_data["quadratic"].toBool();
    // another forward may have replaced the context's image since
    upload(ctx, def_image);
    torch::Tensor rows = rows_for(ctx, params, quadratic);
    torch::Tensor seed = grad_out[0].to(torch::kFloat64).contiguous();
    torch::Tensor dparams = torch::empty({params.size(0), 12}, rows.options());
    torch::Tensor ddef;
    const bool want_def = actx->needs_input_grad(1);
    if (want_def) ddef = torch::zeros_like(def_image, def_image.options().dtype(torch::kFloat32));
    check(dicegpu_adjoint(ctx, rows.data_ptr<double>(), seed.data_ptr<double>(), (int)objective, 0,
                          nullptr, dparams.data_ptr<double>(), want_def ? ddef.data_ptr<float>() : nullptr),
          "adjoint (backward)");
    torch::Tensor gparams = dparams.narrow(1, 0, params.size(1)).to(params.dtype());
    return {gparams, want_def ? ddef.to(def_image.dtype()) : torch::Tensor(), torch::Tensor(),
            torch::Tensor(), torch::Tensor()};
  }
};

torch::Tensor subset_objective(torch::Tensor params, torch::Tensor def_image, int64_t handle,
                               int64_t objective, bool quadratic) {
  return SubsetObjective::apply(params, def_image, handle, objective, quadratic);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("subset_objective", &subset_objective,
        "Per-subset objective (0 gamma, 1 least squares) with an adjoint backward",
        py::arg("params"), py::arg("def_image"), py::arg("ctx"), py::arg("objective") = 0,
        py::arg("quadratic") = false);
}
