// libtorch autograd functions over the gvx C ABI (include/gvx.h):
//   TrilinearDistance : points [N,3] (metres) -> trilinear EDT distance [N]
//   TrajectoryCost    : joint waypoints [B,T,J] -> hinge obstacle cost [B]
// Both backward passes are the hand-written adjoint kernels
// (gvx_query_trilinear_bwd, gvx_traj_cost_bwd); nothing but the inputs is
// saved -- the adjoints recompute the gathers and the forward kinematics.
// Kernels run on the current CUDA stream of the calling thread.
#include <c10/cuda/CUDAStream.h>
#include <torch/extension.h>

#include <cstring>

#include "../../include/gvx.h"

namespace {

using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

void check(gvx_status st) { TORCH_CHECK(st == GVX_OK, "gvx: ", gvx_last_error()); }

gvx_stream current_stream() { return reinterpret_cast<gvx_stream>(c10::cuda::getCurrentCUDAStream().stream()); }

const gvx_dvm* as_map(int64_t handle) {
  TORCH_CHECK(handle != 0, "null map handle");
  return reinterpret_cast<const gvx_dvm*>(handle);
}

gvx_arm unpack_arm(const torch::Tensor& blob) {
  TORCH_CHECK(blob.device().is_cpu() && blob.dtype() == torch::kUInt8 && blob.numel() == (int64_t)sizeof(gvx_arm),
              "arm must be a CPU uint8 tensor holding one gvx_arm");
  gvx_arm arm;
  std::memcpy(&arm, blob.contiguous().data_ptr<uint8_t>(), sizeof(gvx_arm));
  return arm;
}

torch::Tensor f32_cuda(const torch::Tensor& t) {
  TORCH_CHECK(t.is_cuda(), "expected a CUDA tensor");
  return t.to(torch::kFloat32).contiguous();
}

struct TrilinearDistance : public torch::autograd::Function<TrilinearDistance> {
  static torch::Tensor forward(AutogradContext* ctx, torch::Tensor points, int64_t map) {
    auto p = f32_cuda(points);
    TORCH_CHECK(p.dim() == 2 && p.size(1) == 3, "points must be [N,3]");
    auto dist = torch::empty({p.size(0)}, p.options());
    check(gvx_query_trilinear(as_map(map), p.data_ptr<float>(), p.size(0), dist.data_ptr<float>(), nullptr,
                              current_stream()));
    ctx->save_for_backward({p});
    ctx->saved_data["map"] = map;
    return dist;
  }
  static tensor_list backward(AutogradContext* ctx, tensor_list grad_out) {
    auto p = ctx->get_saved_variables()[0];
    auto g = f32_cuda(grad_out[0]);
    auto gp = torch::empty_like(p);
    check(gvx_query_trilinear_bwd(as_map(ctx->saved_data["map"].toInt()), p.data_ptr<float>(), p.size(0),
                                  g.data_ptr<float>(), gp.data_ptr<float>(), current_stream()));
    return {gp, torch::Tensor()};
  }
};

struct TrajectoryCost : public torch::autograd::Function<TrajectoryCost> {
  static torch::Tensor forward(AutogradContext* ctx, torch::Tensor q, int64_t map, torch::Tensor arm_blob, double margin) {
    auto qq = f32_cuda(q);
    const gvx_arm arm = unpack_arm(arm_blob);
    TORCH_CHECK(qq.dim() == 3 && qq.size(2) == arm.n_joints, "q must be [B,T,n_joints]");
    auto cost = torch::empty({qq.size(0)}, qq.options());
    check(gvx_traj_cost(as_map(map), &arm, qq.data_ptr<float>(), qq.size(0), (uint32_t)qq.size(1), (float)margin,
                        cost.data_ptr<float>(), current_stream()));
    ctx->save_for_backward({qq});
    ctx->saved_data["map"] = map;
    ctx->saved_data["arm"] = arm_blob;
    ctx->saved_data["margin"] = margin;
    return cost;
  }
  static tensor_list backward(AutogradContext* ctx, tensor_list grad_out) {
    auto qq = ctx->get_saved_variables()[0];
    const gvx_arm arm = unpack_arm(ctx->saved_data["arm"].toTensor());
    auto g = f32_cuda(grad_out[0]);
    auto gq = torch::empty_like(qq);
    check(gvx_traj_cost_bwd(as_map(ctx->saved_data["map"].toInt()), &arm, qq.data_ptr<float>(), qq.size(0),
                            (uint32_t)qq.size(1), (float)ctx->saved_data["margin"].toDouble(), g.data_ptr<float>(),
                            gq.data_ptr<float>(), current_stream()));
    return {gq, torch::Tensor(), torch::Tensor(), torch::Tensor()};
  }
};

torch::Tensor trilinear_distance(torch::Tensor points, int64_t map) { return TrilinearDistance::apply(points, map); }

torch::Tensor trajectory_cost(torch::Tensor q, int64_t map, torch::Tensor arm_blob, double margin) {
  return TrajectoryCost::apply(q, map, arm_blob, margin);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "gvx autograd functions (hand-written adjoint kernels behind torch::autograd::Function)";
  m.def("trilinear_distance", &trilinear_distance, "trilinear EDT distance with adjoint", py::arg("points"), py::arg("map"));
  m.def("trajectory_cost", &trajectory_cost, "hinge trajectory cost with adjoint", py::arg("q"), py::arg("map"),
        py::arg("arm"), py::arg("margin"));
}
