// Shared plumbing of the C++ drop-in classes (zldsp_fft_cfft.hpp,
// zldsp_fft_rfft.hpp): an owning plan handle over the C ABI of
// libzlfft_cuda and the error policy. The reference's member functions return
// void and have no error channel; these throw std::runtime_error with the
// library's message when a call fails (bad size, CUDA failure).
#pragma once

#include <stdexcept>
#include <string>
#include <type_traits>

#include "../zlfft.h"

namespace zldsp::fft::cuda_detail {

inline void check(int rc) {
    if (rc != ZLFFT_OK) throw std::runtime_error(std::string("zlfft: ") + zlfft_last_error());
}

template <typename F>
constexpr int precision() {
    static_assert(std::is_same_v<F, float> || std::is_same_v<F, double>, "CFFT/RFFT are defined for float and double");
    return std::is_same_v<F, float> ? ZLFFT_F32 : ZLFFT_F64;
}

// Move-only owner of one zlfft plan (the reference objects are move-only too:
// they own hwy::AlignedFreeUniquePtr buffers). Like the reference's
// constructors, the plan picks its algorithm from this host's cache sizes
// (ZLFFT_MODE_HOST: src/common/zldsp_fft_common_init.hpp:305-339), so the
// results are the ones the reference gives on this host.
class Plan {
public:
    Plan(int kind, int precision, size_t order) { check(zlfft_plan_create(&h_, kind, precision, order, ZLFFT_MODE_HOST, -1)); }
    ~Plan() { zlfft_plan_destroy(h_); }
    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;
    Plan(Plan&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    Plan& operator=(Plan&& o) noexcept {
        if (this != &o) {
            zlfft_plan_destroy(h_);
            h_ = o.h_;
            o.h_ = nullptr;
        }
        return *this;
    }
    zlfft_plan get() const { return h_; }
    size_t size() const {
        size_t n = 0;
        check(zlfft_plan_get_size(h_, &n));
        return n;
    }
    size_t order() const {
        size_t o = 0;
        check(zlfft_plan_get_order(h_, &o));
        return o;
    }

private:
    zlfft_plan h_ = nullptr;
};

}  // namespace zldsp::fft::cuda_detail
