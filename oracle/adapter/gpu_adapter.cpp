// The device context the adapter's classes share (one per process, device 0).
#include "gpu_adapter.h"
#include <hist/distance_calculator/SimpleCalculator.h>

#include <mutex>

namespace ausaxs::hist::distance_calculator {
inline namespace gpu {
    ausaxs_gpu_ctx* adapter_context() {
        static std::once_flag once;
        static ausaxs_gpu_ctx* ctx = nullptr;
        std::call_once(once, [] { adapter_check(ausaxs_gpu_ctx_create(0, &ctx)); });
        return ctx;
    }
}
}
