// cufsp_rtc.cu -- run-time compilation of the network-specialised kernels (plane kernel of the
// KRONECKER format, sparse-format kernel) for sm_100a with NVRTC, loaded with cudaLibraryLoadData.
// Compiled modules are cached per process by their full source text, so generators of the same
// network (and, where the box is part of the source, the same box) reuse them.
#include <nvrtc.h>

#include <map>
#include <memory>
#include <mutex>

#include "cufsp_internal.h"

namespace cufsp {

namespace {
std::mutex g_rtc_mu;
std::map<std::string, std::shared_ptr<RtcModule>> g_rtc_cache;
}  // namespace

std::shared_ptr<RtcModule> rtc_module(const std::string &src, const std::vector<std::string> &names, std::string &why) {
    std::lock_guard<std::mutex> lock(g_rtc_mu);
    std::string key = src;
    for (const auto &n : names) key += "\n//kernel " + n;
    auto it = g_rtc_cache.find(key);
    if (it != g_rtc_cache.end()) return it->second;
    auto mod = std::make_shared<RtcModule>();
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "cufsp_rtc.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        why = "nvrtcCreateProgram failed";
        return nullptr;
    }
    const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=true", "-lineinfo"};
    const nvrtcResult rc = nvrtcCompileProgram(prog, 4, opts);
    size_t log_size = 0;
    nvrtcGetProgramLogSize(prog, &log_size);
    if (log_size > 1) {
        mod->log.resize(log_size);
        nvrtcGetProgramLog(prog, &mod->log[0]);
    }
    if (rc != NVRTC_SUCCESS) {
        why = std::string("NVRTC: ") + nvrtcGetErrorString(rc) + ": " + mod->log.substr(0, 2000);
        nvrtcDestroyProgram(&prog);
        return nullptr;
    }
    size_t cubin_size = 0;
    std::vector<char> cubin;
    if (nvrtcGetCUBINSize(prog, &cubin_size) == NVRTC_SUCCESS && cubin_size > 0) {
        cubin.resize(cubin_size);
        if (nvrtcGetCUBIN(prog, cubin.data()) != NVRTC_SUCCESS) cubin.clear();
    }
    nvrtcDestroyProgram(&prog);
    if (cubin.empty()) {
        why = "NVRTC produced no cubin";
        return nullptr;
    }
    cudaError_t e = cudaLibraryLoadData(&mod->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    for (const auto &n : names) {
        cudaKernel_t k = nullptr;
        if (e == cudaSuccess) e = cudaLibraryGetKernel(&k, mod->lib, n.c_str());
        mod->kernels.push_back(k);
    }
    if (e != cudaSuccess) {
        why = std::string("loading the run-time compiled kernels: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return nullptr;
    }
    g_rtc_cache[key] = mod;
    return mod;
}

}  // namespace cufsp
