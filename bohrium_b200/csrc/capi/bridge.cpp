// The flat C bridge declared in include/bh_b200.h.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <bh_b200.h>
#include <bohrium/bh_component.hpp>
#include <bohrium/bh_main_memory.hpp>
#include <map>
#include <sstream>
#include "../core/filters.hpp"

using namespace std;
using namespace bohrium;

namespace {
thread_local string g_last_error;

template <typename F>
int guarded(F &&f) {
    try {
        f();
        g_last_error.clear();
        return 0;
    } catch (const std::exception &e) {
        g_last_error = e.what();
    } catch (...) {
        g_last_error = "unknown error";
    }
    return -1;
}
} // namespace

struct bhb_runtime {
    unique_ptr<ConfigParser> config;
    component::ComponentFace child;
    string message;
};

struct bhb_ir {
    ~bhb_ir() {
        if (ir) bh_ir_hints_clear(ir.get());
    }
    unique_ptr<BhIR> ir;
    bohrium::filter::BaseStore created;  // temporaries made by bhb_ir_filter
    string text;                          // last bhb_ir_text result
};

namespace {
// Content fingerprint of a decoded list without sliding views: every instruction's opcode,
// constant and operand views, with each base's address, element type and size (an address can be
// reused for another base), plus the syncs and repeat settings. Never 0.
uint64_t fingerprint(const BhIR &ir) {
    uint64_t h = 0xcbf29ce484222325ULL ^ static_cast<uint64_t>(ir.instr_list.size());
    auto mix = [&h](uint64_t v) {
        v *= 0x9E3779B97F4A7C15ULL;
        h = (h ^ (v ^ (v >> 29))) * 0x100000001B3ULL;
    };
    for (const bh_instruction &instr : ir.instr_list) {
        mix(static_cast<uint64_t>(instr.opcode));
        mix(static_cast<uint64_t>(instr.constant.type));
        uint64_t cw[2] = {0, 0};
        memcpy(cw, &instr.constant.value, min(sizeof(cw), sizeof(instr.constant.value)));
        mix(cw[0]);
        mix(cw[1]);
        mix(instr.operand.size());
        for (const bh_view &v : instr.operand) {
            if (v.isConstant()) {
                mix(~0ULL);
                continue;
            }
            mix(reinterpret_cast<uint64_t>(v.base));
            mix(static_cast<uint64_t>(v.base->dtype()));
            mix(static_cast<uint64_t>(v.base->nelem()));
            mix(static_cast<uint64_t>(v.start));
            mix(static_cast<uint64_t>(v.ndim));
            for (int64_t d = 0; d < v.ndim; ++d) {
                mix(static_cast<uint64_t>(v.shape[d]));
                mix(static_cast<uint64_t>(v.stride[d]));
            }
        }
    }
    for (const bh_base *b : ir._syncs) mix(reinterpret_cast<uint64_t>(b));
    mix(ir._nrepeats);
    mix(reinterpret_cast<uint64_t>(ir._repeat_condition));
    return h | 1ULL;
}

BhIR *decode(const int64_t *w, int64_t n, bh_base *const *syncs, int64_t nsyncs, uint64_t nrepeats, bh_base *cond,
             const int64_t *slides, int64_t nslide) {
    vector<bh_instruction> list;
    int64_t i = 0;
    auto need = [&](int64_t k) {
        if (i + k > n) throw runtime_error("bhb: truncated instruction encoding");
    };
    while (i < n) {
        need(5);
        bh_instruction instr;
        instr.opcode = w[i];
        const int64_t nop = w[i + 1];
        const int64_t ctype = w[i + 2];
        if (nop < 0 || nop > 8) throw runtime_error("bhb: bad operand count");
        if (ctype >= 0) {
            if (ctype >= BH_NUM_TYPES) throw runtime_error("bhb: bad constant type");
            instr.constant.type = static_cast<bh_type>(ctype);
            memcpy(&instr.constant.value, &w[i + 3], 16);
        } else {
            instr.constant.type = bh_type::BOOL;
            memset(&instr.constant.value, 0, 16);
        }
        i += 5;
        for (int64_t o = 0; o < nop; ++o) {
            need(1);
            bh_view v;
            v.base = reinterpret_cast<bh_base *>(w[i++]);
            if (v.base != nullptr) {
                need(2);
                v.start = w[i];
                v.ndim = w[i + 1];
                i += 2;
                if (v.ndim < 0 || v.ndim > BH_MAXDIM) throw runtime_error("bhb: bad ndim");
                need(2 * v.ndim);
                v.shape.resize(static_cast<size_t>(v.ndim));
                v.stride.resize(static_cast<size_t>(v.ndim));
                for (int64_t d = 0; d < v.ndim; ++d) v.shape[d] = w[i + d];
                for (int64_t d = 0; d < v.ndim; ++d) v.stride[d] = w[i + v.ndim + d];
                i += 2 * v.ndim;
            }
            instr.operand.push_back(v);
        }
        if (instr.opcode <= BH_MAX_OPCODE_ID) {
            const int expect = bh_opcode_nop(instr.opcode);
            if (expect < 0) throw runtime_error("bhb: unknown opcode " + to_string(instr.opcode));
            if (expect != static_cast<int>(nop))
                throw runtime_error(string("bhb: ") + bh_opcode_text(instr.opcode) + " expects " + to_string(expect) +
                                    " operands");
        }
        list.push_back(std::move(instr));
    }
    // Sliding views
    int64_t j = 0;
    while (j < nslide) {
        const int64_t ii = slides[j], oo = slides[j + 1], nd = slides[j + 2];
        j += 3;
        if (ii < 0 || ii >= static_cast<int64_t>(list.size()) || oo < 0 ||
            oo >= static_cast<int64_t>(list[ii].operand.size()))
            throw runtime_error("bhb: bad slide target");
        bh_view &v = list[ii].operand[oo];
        for (int64_t d = 0; d < nd; ++d) {
            bh_slide_dim sd{slides[j], slides[j + 1], slides[j + 2], slides[j + 3], slides[j + 4], slides[j + 5]};
            v.slides.dims.push_back(sd);
            j += 6;
        }
        const int64_t nr = slides[j++];
        for (int64_t r = 0; r < nr; ++r) {
            v.slides.resets[slides[j]] = make_pair(slides[j + 1], int64_t{0});
            j += 2;
        }
    }
    bool builtin = true;
    for (const bh_instruction &instr : list) builtin = builtin && instr.opcode <= BH_MAX_OPCODE_ID;
    set<bh_base *> s(syncs, syncs + nsyncs);
    BhIR *ir = new BhIR(std::move(list), std::move(s), nrepeats, cond);
    BhIRHints hints;
    hints.plain = nslide == 0 && builtin;
    // Sliding views change between executions, so such a list gets no fingerprint.
    if (nslide == 0) hints.fingerprint = fingerprint(*ir);
    bh_ir_hints_set(ir, hints);
    return ir;
}
} // namespace

extern "C" {

const char *bhb_last_error(void) { return g_last_error.c_str(); }

bhb_runtime *bhb_runtime_create(const char *config_path, const char *stack_name) {
    bhb_runtime *rt = nullptr;
    guarded([&] {
        // Components below the bridge locate the config themselves, as in the reference.
        if (config_path && config_path[0]) setenv("BH_CONFIG", config_path, 1);
        if (stack_name && stack_name[0]) setenv("BH_STACK", stack_name, 1);
        unique_ptr<bhb_runtime> r(new bhb_runtime());
        r->config.reset(new ConfigParser(-1));
        const string child = r->config->getChildLibraryPath();
        if (child.empty()) throw runtime_error("bhb_runtime_create: the stack is empty");
        r->child = component::ComponentFace(child, 0);
        rt = r.release();
    });
    return rt;
}

void bhb_runtime_destroy(bhb_runtime *rt) {
    guarded([&] { delete rt; });
}

bh_base *bhb_base_create(int dtype, int64_t nelem) {
    bh_base *b = nullptr;
    guarded([&] {
        if (dtype < 0 || dtype >= BH_NUM_TYPES) throw runtime_error("bhb_base_create: bad dtype");
        if (nelem < 0) throw runtime_error("bhb_base_create: negative size");
        b = new bh_base(nelem, static_cast<bh_type>(dtype));
    });
    return b;
}

void bhb_base_destroy(bh_base *base) { delete base; }
int bhb_base_dtype(const bh_base *base) { return static_cast<int>(base->dtype()); }
int64_t bhb_base_nelem(const bh_base *base) { return base->nelem(); }

void *bhb_data_get(bhb_runtime *rt, bh_base *base, int copy2host, int force_alloc, int nullify) {
    void *ret = nullptr;
    guarded([&] { ret = rt->child.getMemoryPointer(*base, copy2host != 0, force_alloc != 0, nullify != 0); });
    return ret;
}

int bhb_data_set(bhb_runtime *rt, bh_base *base, int host_ptr, void *data) {
    return guarded([&] { rt->child.setMemoryPointer(base, host_ptr != 0, data); });
}

void *bhb_host_alloc(bhb_runtime *rt, int64_t nbytes) {
    void *ret = nullptr;
    guarded([&] {
        const string r = rt->child.message("host_alloc " + to_string(nbytes));
        ret = reinterpret_cast<void *>(strtoull(r.c_str(), nullptr, 10));
        if (ret == nullptr) ret = malloc(static_cast<size_t>(nbytes));
        if (ret == nullptr) throw bad_alloc();
    });
    return ret;
}

int bhb_data_copy_in(bhb_runtime *rt, bh_base *base, const void *src, int64_t nbytes) {
    return guarded([&] {
        if (nbytes != base->nbytes()) throw runtime_error("bhb_data_copy_in: size mismatch");
        void *p = rt->child.getMemoryPointer(*base, true, true, false);
        if (nbytes > 0) memcpy(p, src, static_cast<size_t>(nbytes));
    });
}

bhb_ir *bhb_ir_create(const int64_t *words, int64_t nwords, bh_base *const *syncs, int64_t nsyncs, uint64_t nrepeats,
                      bh_base *repeat_condition, const int64_t *slides, int64_t nslide_words) {
    bhb_ir *ret = nullptr;
    guarded([&] {
        unique_ptr<bhb_ir> r(new bhb_ir());
        r->ir.reset(decode(words, nwords, syncs, nsyncs, nrepeats, repeat_condition, slides, nslide_words));
        ret = r.release();
    });
    return ret;
}

void bhb_ir_destroy(bhb_ir *ir) { delete ir; }

int bhb_ir_execute(bhb_runtime *rt, bhb_ir *ir) {
    return guarded([&] { rt->child.execute(ir->ir.get()); });
}

int bhb_execute(bhb_runtime *rt, const int64_t *words, int64_t nwords, bh_base *const *syncs, int64_t nsyncs,
                uint64_t nrepeats, bh_base *repeat_condition, const int64_t *slides, int64_t nslide_words) {
    return guarded([&] {
        unique_ptr<BhIR> ir(decode(words, nwords, syncs, nsyncs, nrepeats, repeat_condition, slides, nslide_words));
        struct Clear {
            const BhIR *p;
            ~Clear() { bh_ir_hints_clear(p); }
        } clear{ir.get()};
        rt->child.execute(ir.get());
    });
}

const char *bhb_message(bhb_runtime *rt, const char *msg) {
    const int r = guarded([&] { rt->message = rt->child.message(msg); });
    return r == 0 ? rt->message.c_str() : nullptr;
}

int bhb_extmethod(bhb_runtime *rt, const char *name, int64_t opcode) {
    return guarded([&] {
        if (opcode <= BH_MAX_OPCODE_ID) throw runtime_error("bhb_extmethod: opcode must be > BH_MAX_OPCODE_ID");
        rt->child.extmethod(name, opcode);
    });
}

const char *bhb_user_kernel(bhb_runtime *rt, const char *kernel, int64_t nop, bh_base *const *operands,
                            const char *compile_cmd, const char *tag, const char *param) {
    const int r = guarded([&] {
        if (kernel == nullptr || tag == nullptr) throw runtime_error("bhb_user_kernel: kernel and tag are required");
        if (nop < 0 || (nop > 0 && operands == nullptr)) throw runtime_error("bhb_user_kernel: bad operand list");
        vector<bh_view> ops;
        for (int64_t i = 0; i < nop; ++i) {
            if (operands[i] == nullptr) throw runtime_error("bhb_user_kernel: null operand");
            ops.emplace_back(operands[i]);
        }
        rt->message = rt->child.userKernel(kernel, ops, compile_cmd ? compile_cmd : "", tag, param ? param : "");
    });
    return r == 0 ? rt->message.c_str() : nullptr;
}

void *bhb_get_device_context(bhb_runtime *rt) {
    void *r = nullptr;
    guarded([&] { r = rt->child.getDeviceContext(); });
    return r;
}

int bhb_set_device_context(bhb_runtime *rt, void *ctx) {
    return guarded([&] { rt->child.setDeviceContext(ctx); });
}

double bhb_last_execute_ms(bhb_runtime *rt) {
    double ms = 0;
    guarded([&] {
        const string r = rt->child.message("CUDA: last execute ms");
        ms = r.empty() ? 0.0 : strtod(r.c_str(), nullptr);
    });
    return ms;
}

} // extern "C"

// Access to the decoded BhIR of a bhb_ir handle (used by in-tree components' test hooks).
extern "C" void *bhb_ir_bhir(bhb_ir *ir) { return ir ? static_cast<void *>(ir->ir.get()) : nullptr; }
extern "C" void bhb_set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

// Host data pointer of a base (valid after a sync; NULL when the base has no host storage).
extern "C" void *bhb_base_data(const bh_base *base) { return const_cast<void *>(base->getDataPtr()); }

// Apply a bytecode filter to a decoded BhIR in place (test hook of the filter components):
// "bcexp" (powk), "bcexp+sign" (powk and sign), "bccon" (stupidmath, collect, muladd). Returns
// the number of rewrites, or -1 on error.
extern "C" int bhb_ir_filter(bhb_ir *ir, const char *name) {
    int n = -1;
    guarded([&] {
        const string f = name ? name : "";
        if (f.compare(0, 5, "bcexp") == 0 && (f.size() == 5 || f[5] == '+')) {
            // "bcexp" with "+"-separated options: "sign", "reduce1d=<thread limit>"
            bohrium::filter::ExpandOptions o;
            size_t pos = 5;
            while (pos < f.size()) {
                const size_t next = f.find('+', pos + 1);
                const string opt = f.substr(pos + 1, next == string::npos ? string::npos : next - pos - 1);
                if (opt == "sign") {
                    o.sign = true;
                } else if (opt.compare(0, 9, "reduce1d=") == 0) {
                    o.reduce1d = stoll(opt.substr(9));
                } else {
                    throw runtime_error("bhb_ir_filter: unknown bcexp option " + opt);
                }
                pos = next == string::npos ? f.size() : next;
            }
            n = bohrium::filter::expand(*ir->ir, o, ir->created);
        } else if (f == "bccon") {
            n = bohrium::filter::contract(*ir->ir, bohrium::filter::ContractOptions());
        } else {
            throw runtime_error("bhb_ir_filter: unknown filter " + f);
        }
        // The list changed: a fingerprint must describe the filtered list.
        BhIRHints hints = bh_ir_hints_get(ir->ir.get());
        if (hints.fingerprint != 0) hints.fingerprint = fingerprint(*ir->ir);
        bh_ir_hints_set(ir->ir.get(), hints);
    });
    return n;
}

// A text listing of a decoded BhIR, one instruction per line: the opcode number, then each
// operand as `c` (the constant) or `b<k>[start;shape;stride]` with bases numbered by first
// appearance, then the constant's value for instructions that have one.
extern "C" const char *bhb_ir_text(bhb_ir *ir) {
    const char *ret = nullptr;
    guarded([&] {
        stringstream ss;
        std::map<const bh_base *, int> ids;
        for (const bh_instruction &in : ir->ir->instr_list) {
            if (in.opcode == BH_NONE) continue;
            ss << in.opcode;
            for (const bh_view &v : in.operand) {
                if (v.isConstant()) {
                    ss << " c";
                    continue;
                }
                auto it = ids.emplace(v.base, static_cast<int>(ids.size())).first;
                ss << " b" << it->second << "[" << v.start << ";";
                for (int64_t d = 0; d < v.ndim; ++d) ss << (d ? "," : "") << v.shape[d];
                ss << ";";
                for (int64_t d = 0; d < v.ndim; ++d) ss << (d ? "," : "") << v.stride[d];
                ss << "]";
            }
            if (in.has_constant()) ss << " = " << in.constant.get_double();
            ss << "\n";
        }
        ir->text = ss.str();
        ret = ir->text.c_str();
    });
    return ret;
}
