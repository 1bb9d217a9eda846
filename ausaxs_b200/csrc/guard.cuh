// Exception-to-status wrapper shared by the C entry points: engine errors become status codes, their
// text is kept for ausaxs_gpu_last_error() (the reference's execute_with_catch,
// include/api/api/api_helper.h:25-45).
#pragma once
#include <exception>

#include "engine.cuh"

namespace ausaxs_b200 {
void set_last_error(const char* msg);  // capi.cu

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return AUSAXS_OK;
    } catch (const Error& e) {
        set_last_error(e.msg.c_str());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return AUSAXS_ERR_CUDA;
    } catch (...) {
        set_last_error("unknown failure");
        return AUSAXS_ERR_CUDA;
    }
}
}  // namespace ausaxs_b200
