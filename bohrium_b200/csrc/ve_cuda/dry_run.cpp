// Device-free inspection of the engine's lowering: fuse a BhIR, generate the kernel sources and
// optionally compile them with NVRTC for sm_100a. Used by the CPU test-suite to check every code
// path up to the launch on a machine without a GPU.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <sstream>
#include <string>
#include <vector>
#include <nvrtc.h>
#include <bh_b200.h>
#include <bohrium/bh_ir.hpp>
#include "../jitk/fuser.hpp"
#include "codegen.hpp"

using namespace std;
using namespace bohrium;

extern "C" void *bhb_ir_bhir(bhb_ir *ir);
extern "C" void bhb_set_last_error(const char *msg);

namespace {
string json_escape(const string &s) {
    string r;
    for (char c : s) {
        switch (c) {
            case '"': r += "\\\""; break;
            case '\\': r += "\\\\"; break;
            case '\n': r += "\\n"; break;
            case '\t': r += "\\t"; break;
            default:
                if (static_cast<unsigned char>(c) < 0x20) {
                    char buf[8];
                    snprintf(buf, sizeof buf, "\\u%04x", static_cast<unsigned>(static_cast<unsigned char>(c)));
                    r += buf;
                } else {
                    r += c;
                }
        }
    }
    return r;
}

string nvrtc_compile(const string &src, const string &name, bool fmad) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), (name + ".cu").c_str(), 0, nullptr, nullptr) != NVRTC_SUCCESS)
        return "nvrtcCreateProgram failed";
    const char *opts[] = {"-arch=sm_100a", "-std=c++17", fmad ? "--fmad=true" : "--fmad=false"};
    const nvrtcResult r = nvrtcCompileProgram(prog, 3, opts);
    string log;
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetProgramLogSize(prog, &n);
        log.assign(n, '\0');
        nvrtcGetProgramLog(prog, &log[0]);
        log = "NVRTC: " + log;
    }
    nvrtcDestroyProgram(&prog);
    return log;
}
} // namespace

// Returns a JSON document (static storage, valid until the next call) describing the kernels
// and launch units of `ir`, or NULL on error (see bhb_last_error()).
// `fuser_list` (comma separated, NULL for the engine default) overrides the transformer list.
extern "C" const char *bh_ve_cuda_dry_run(bhb_ir *handle, int compile, const char *fuser_list) {
    static string out;
    try {
        BhIR &bhir = *static_cast<BhIR *>(bhb_ir_bhir(handle));
        vector<bh_instruction> copy = bhir.instr_list;
        cuda::contract_multiply_add(copy, bhir._syncs);
        set<bh_base *> frees;
        vector<bh_instruction *> instr_list = jitk::remove_non_computed_system_instr(copy, frees);
        set<const bh_base *> constructed;
        for (bh_instruction *instr : instr_list) {
            instr->constructor = false;
            for (size_t o = 0; o < instr->operand.size(); ++o) {
                const bh_view &v = instr->operand[o];
                if (v.isConstant()) continue;
                if (o == 0 && !constructed.count(v.base) && v.base->getDataPtr() == nullptr) instr->constructor = true;
                constructed.insert(v.base);
            }
        }
        jitk::FusionConfig cfg;
        cfg.fuser_list = {"greedy", "push_reductions_inwards", "collapse_redundant_axes"};
        if (fuser_list != nullptr && fuser_list[0]) {
            cfg.fuser_list.clear();
            string cur;
            for (const char *p = fuser_list;; ++p) {
                if (*p == ',' || *p == ' ' || *p == '\0') {
                    if (!cur.empty()) cfg.fuser_list.push_back(cur);
                    cur.clear();
                    if (*p == '\0') break;
                } else {
                    cur += *p;
                }
            }
        }
        // The engine's defaults (bohrium_b200/config.ini).
        cfg.avoid_rank0_sweep = false;
        cfg.avoid_mixed_sweeps = true;
        const vector<jitk::LoopB> kernels = jitk::get_kernel_list(instr_list, cfg);
        cuda::CodegenOptions opt;
        // The engine's codegen keys, from the environment as the config would give them.
        if (const char *v = getenv("BH_CUDA_INTERLEAVE")) opt.interleave = atoi(v);
        if (const char *v = getenv("BH_CUDA_PRELOAD_HEAVY")) opt.preload_heavy = string(v) == "true" || string(v) == "1";
        if (const char *v = getenv("BH_CUDA_TILE2D")) opt.tile2d = string(v) == "true" || string(v) == "1";
        if (const char *v = getenv("BH_CUDA_VECTOR_ACCESS")) opt.vector_access = string(v) == "true" || string(v) == "1";
        if (const char *v = getenv("BH_CUDA_SCAN_SINGLE_PASS")) opt.scan_single_pass = string(v) == "true" || string(v) == "1";
        if (const char *v = getenv("BH_CUDA_SCAN_WINDOWS")) opt.scan_windows = string(v) == "true" || string(v) == "1";
        if (const char *v = getenv("BH_CUDA_STAGE_BULK")) opt.stage_bulk = string(v) == "true" || string(v) == "1";
        if (const char *v = getenv("BH_CUDA_SCAN_PREFETCH")) opt.scan_prefetch = string(v) == "true" || string(v) == "1";
        vector<vector<cuda::LaunchUnit>> lowered(kernels.size());
        for (size_t k = 0; k < kernels.size(); ++k)
            if (!kernels[k].isSystemOnly()) lowered[k] = cuda::lower_kernel(kernels[k], opt);
        const vector<int> folded = cuda::fuse_tails(kernels, lowered, opt);
        stringstream ss;
        ss << "{\"kernels\": [";
        for (size_t k = 0; k < kernels.size(); ++k) {
            if (k) ss << ", ";
            ss << "{\"block\": \"" << json_escape(kernels[k].pprint()) << "\", \"folded_into\": " << folded[k]
               << ", \"units\": [";
            const vector<cuda::LaunchUnit> &units = lowered[k];
            for (size_t u = 0; u < units.size(); ++u) {
                if (u) ss << ", ";
                string err;
                if (compile) err = nvrtc_compile(units[u].source, units[u].name, false);
                ss << "{\"name\": \"" << units[u].name << "\", \"sched\": \"" << cuda::sched_name(units[u].sched)
                   << "\", \"fields\": " << units[u].fields.size() << ", \"work\": " << units[u].work_items()
                   << ", \"bytes\": " << units[u].algorithmic_bytes << ", \"tail\": " << (units[u].tail ? "true" : "false")
                   << ", \"compile_error\": \"" << json_escape(err)
                   << "\", \"source\": \"" << json_escape(units[u].source) << "\"}";
            }
            ss << "]}";
        }
        ss << "]}";
        out = ss.str();
        return out.c_str();
    } catch (const std::exception &e) {
        bhb_set_last_error(e.what());
        return nullptr;
    }
}
