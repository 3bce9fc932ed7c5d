// libtorch autograd Functions of the differentiable receive path (extension without a reference
// counterpart), registered as torch.ops.supra_b200.das_apod and torch.ops.supra_b200.envelope.
//
// Forward and backward both call the C ABI of libsupra_b200.so on the current CUDA stream:
// sb_das_forward_apod / sb_das_adjoint (gradients w.r.t. channel data, per-element apodisation and
// speed of sound; aperture tiles are recomputed in the backward pass, only the forward output is
// saved) and sb_hilbert_env_run / sb_hilbert_env_adjoint. The DAS plan and the Hilbert plan are
// passed as integer handles (sb_das_plan*, sb_hilbert_plan*) owned by the caller.
#include <ATen/cuda/CUDAContext.h>
#include <torch/autograd.h>
#include <torch/types.h>
#include <torch/library.h>

#include <string>

#include "supra_b200.h"

namespace {

using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

void check(const char* fn, int status) {
    TORCH_CHECK(status == SB_OK, fn, " failed with status ", status, ": ", sb_last_error());
}

sb_stream currentStream() { return reinterpret_cast<sb_stream>(at::cuda::getCurrentCUDAStream().stream()); }

const float* ptrOrNull(const torch::Tensor& t) { return t.defined() ? t.data_ptr<float>() : nullptr; }

class DasApodFn : public torch::autograd::Function<DasApodFn> {
public:
    // rf [frames][tx][channels][samples] FP32 CUDA, apod [elements] (undefined = 1), c: 0-dim (mm/s)
    static torch::Tensor forward(AutogradContext* ctx, torch::Tensor rf, torch::Tensor apod, torch::Tensor c, int64_t plan,
                                 int64_t numDepths, int64_t numRx, double fNumber, int64_t windowType, double windowParameter) {
        TORCH_CHECK(rf.is_cuda() && rf.scalar_type() == torch::kFloat32 && rf.dim() == 4, "rf: CUDA float32 [F][tx][ch][samples]");
        rf = rf.contiguous();
        if (apod.defined()) apod = apod.contiguous();
        const double cv = c.item<double>();
        auto out = torch::empty({rf.size(0), numDepths, numRx}, rf.options());
        check("sb_das_forward_apod",
              sb_das_forward_apod(reinterpret_cast<const sb_das_plan*>(plan), rf.data_ptr<float>(), ptrOrNull(apod),
                                  out.data_ptr<float>(), static_cast<uint32_t>(rf.size(0)), fNumber, cv,
                                  static_cast<int>(windowType), static_cast<float>(windowParameter), currentStream()));
        ctx->save_for_backward({rf, apod, out});
        ctx->saved_data["plan"] = plan;
        ctx->saved_data["c"] = cv;
        ctx->saved_data["fNumber"] = fNumber;
        ctx->saved_data["windowType"] = windowType;
        ctx->saved_data["windowParameter"] = windowParameter;
        ctx->saved_data["cDtype"] = static_cast<int64_t>(c.scalar_type());
        ctx->saved_data["cDevice"] = c.device();
        return out;
    }

    static tensor_list backward(AutogradContext* ctx, tensor_list grads) {
        const auto saved = ctx->get_saved_variables();
        const torch::Tensor rf = saved[0], apod = saved[1], out = saved[2];
        const torch::Tensor g = grads[0].contiguous();
        const bool needRf = ctx->needs_input_grad(0), needApod = ctx->needs_input_grad(1) && apod.defined(),
                   needC = ctx->needs_input_grad(2);
        torch::Tensor gRf = needRf ? torch::empty_like(rf) : torch::Tensor();
        torch::Tensor gAp = needApod ? torch::empty_like(apod) : torch::Tensor();
        torch::Tensor gC = needC ? torch::empty({1}, rf.options()) : torch::Tensor();
        check("sb_das_adjoint",
              sb_das_adjoint(reinterpret_cast<const sb_das_plan*>(ctx->saved_data["plan"].toInt()), rf.data_ptr<float>(),
                             ptrOrNull(apod), out.data_ptr<float>(), g.data_ptr<float>(),
                             needRf ? gRf.data_ptr<float>() : nullptr, needApod ? gAp.data_ptr<float>() : nullptr,
                             needC ? gC.data_ptr<float>() : nullptr, static_cast<uint32_t>(rf.size(0)),
                             ctx->saved_data["fNumber"].toDouble(), ctx->saved_data["c"].toDouble(),
                             static_cast<int>(ctx->saved_data["windowType"].toInt()),
                             static_cast<float>(ctx->saved_data["windowParameter"].toDouble()), currentStream()));
        if (needC)
            gC = gC.reshape({}).to(ctx->saved_data["cDevice"].toDevice(),
                                   static_cast<c10::ScalarType>(ctx->saved_data["cDtype"].toInt()));
        return {gRf, gAp, gC, torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor(),
                torch::Tensor()};
    }
};

class EnvelopeFn : public torch::autograd::Function<EnvelopeFn> {
public:
    // img [..., samples, scanlines] FP32 CUDA; every leading index is one image
    static torch::Tensor forward(AutogradContext* ctx, torch::Tensor img, int64_t hilbertPlan) {
        TORCH_CHECK(img.is_cuda() && img.scalar_type() == torch::kFloat32 && img.dim() >= 2, "img: CUDA float32 [..., S, L]");
        img = img.contiguous();
        auto out = torch::empty_like(img);
        const int64_t nS = img.size(-2), nL = img.size(-1), n = img.numel() / (nS * nL);
        for (int64_t i = 0; i < n; i++)
            check("sb_hilbert_env_run",
                  sb_hilbert_env_run(reinterpret_cast<const sb_hilbert_plan*>(hilbertPlan), img.data_ptr<float>() + i * nS * nL,
                                     SB_FLOAT32, out.data_ptr<float>() + i * nS * nL, SB_FLOAT32, static_cast<uint32_t>(nL),
                                     static_cast<uint32_t>(nS), currentStream()));
        ctx->save_for_backward({img});
        ctx->saved_data["plan"] = hilbertPlan;
        return out;
    }

    static tensor_list backward(AutogradContext* ctx, tensor_list grads) {
        const torch::Tensor img = ctx->get_saved_variables()[0];
        const torch::Tensor g = grads[0].contiguous();
        auto gi = torch::empty_like(img);
        const int64_t nS = img.size(-2), nL = img.size(-1), n = img.numel() / (nS * nL);
        for (int64_t i = 0; i < n; i++)
            check("sb_hilbert_env_adjoint",
                  sb_hilbert_env_adjoint(reinterpret_cast<const sb_hilbert_plan*>(ctx->saved_data["plan"].toInt()),
                                         img.data_ptr<float>() + i * nS * nL, g.data_ptr<float>() + i * nS * nL,
                                         gi.data_ptr<float>() + i * nS * nL, static_cast<uint32_t>(nL),
                                         static_cast<uint32_t>(nS), currentStream()));
        return {gi, torch::Tensor()};
    }
};

torch::Tensor dasApod(torch::Tensor rf, std::optional<torch::Tensor> apod, torch::Tensor c, int64_t plan, int64_t numDepths,
                      int64_t numRx, double fNumber, int64_t windowType, double windowParameter) {
    return DasApodFn::apply(rf, apod.has_value() ? *apod : torch::Tensor(), c, plan, numDepths, numRx, fNumber, windowType,
                            windowParameter);
}

torch::Tensor envelope(torch::Tensor img, int64_t hilbertPlan) { return EnvelopeFn::apply(img, hilbertPlan); }

}  // namespace

TORCH_LIBRARY(supra_b200, m) {
    m.def("das_apod(Tensor rf, Tensor? apod, Tensor c, int plan, int num_depths, int num_rx, float f_number, "
          "int window_type, float window_parameter) -> Tensor",
          &dasApod);
    m.def("envelope(Tensor img, int hilbert_plan) -> Tensor", &envelope);
}
