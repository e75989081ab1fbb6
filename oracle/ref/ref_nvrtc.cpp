// Compiles one of the reference's kernel modules the way the reference does at
// run time (src/cuda/CudaModularProgram.cpp:282-304 options, :384-430 link):
// NVRTC to LTO IR (or PTX), then nvJitLink to a cubin for sm_100. Test
// infrastructure: the cubin runs only as the reference in parity checks.
//
//   ref_nvrtc <module.cu> <out.cubin> <kernel_root> <project_include> <variant>
//
// variant "shipped": the reference's options verbatim (--use_fast_math, -dlto).
// variant "ieee":    the same without --use_fast_math, with --fmad=false, PTX link.
#include <nvJitLink.h>
#include <nvrtc.h>

#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

static std::string readFile(const std::string& p) {
    std::ifstream f(p, std::ios::binary);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: ref_nvrtc module.cu out.cubin kernel_root project_include shipped|ieee\n");
        return 2;
    }
    const std::string mod = argv[1], out = argv[2], kroot = argv[3], pinc = argv[4], variant = argv[5];
    const bool ieee = variant == "ieee";
    const std::string src = readFile(mod);
    if (src.empty()) {
        std::fprintf(stderr, "cannot read %s\n", mod.c_str());
        return 1;
    }
    const std::string dir = mod.substr(0, mod.find_last_of('/'));
    const std::string cuda = "/usr/local/cuda/include";
    std::vector<std::string> opts = {"--gpu-architecture=compute_100",
                                     "--extra-device-vectorization",
                                     "-lineinfo",
                                     "-I" + cuda,
                                     "-I" + cuda + "/cccl",
                                     "-I" + dir,
                                     "-I" + kroot,
                                     "-I" + pinc,
                                     "--relocatable-device-code=true",
                                     "-default-device",
                                     "--std=c++20",
                                     "--disable-warnings"};
    if (ieee) {
        opts.push_back("--fmad=false");
    } else {
        opts.push_back("--use_fast_math");
        opts.push_back("-dlto");
    }
    std::vector<const char*> copts;
    for (auto& o : opts) copts.push_back(o.c_str());
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), mod.c_str(), 0, nullptr, nullptr) != NVRTC_SUCCESS) return 1;
    nvrtcResult r = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        nvrtcGetProgramLog(prog, &log[0]);
        std::fprintf(stderr, "compile failed: %s\n%s\n", mod.c_str(), log.c_str());
        return 1;
    }
    std::vector<char> image;
    size_t sz = 0;
    if (ieee) {
        nvrtcGetPTXSize(prog, &sz);
        image.resize(sz);
        nvrtcGetPTX(prog, image.data());
    } else {
        nvrtcGetLTOIRSize(prog, &sz);
        image.resize(sz);
        nvrtcGetLTOIR(prog, image.data());
    }
    nvrtcDestroyProgram(&prog);

    std::vector<const char*> lopts;
    if (!ieee) lopts.push_back("-dlto");
    lopts.push_back("-arch=sm_100");
    nvJitLinkHandle h;
    if (nvJitLinkCreate(&h, (uint32_t)lopts.size(), lopts.data()) != NVJITLINK_SUCCESS) return 1;
    if (nvJitLinkAddData(h, ieee ? NVJITLINK_INPUT_PTX : NVJITLINK_INPUT_LTOIR, image.data(), image.size(),
                         mod.c_str()) != NVJITLINK_SUCCESS ||
        nvJitLinkComplete(h) != NVJITLINK_SUCCESS) {
        size_t n = 0;
        nvJitLinkGetErrorLogSize(h, &n);
        std::string log(n, '\0');
        if (n) nvJitLinkGetErrorLog(h, &log[0]);
        std::fprintf(stderr, "link failed: %s\n%s\n", mod.c_str(), log.c_str());
        return 1;
    }
    size_t csz = 0;
    nvJitLinkGetLinkedCubinSize(h, &csz);
    std::vector<char> cubin(csz);
    nvJitLinkGetLinkedCubin(h, cubin.data());
    nvJitLinkDestroy(&h);
    std::ofstream f(out, std::ios::binary);
    f.write(cubin.data(), (std::streamsize)cubin.size());
    return f.good() ? 0 : 1;
}
