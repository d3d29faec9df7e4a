// The Bohrium Internal Representation: one flushed batch of instructions.
// Fields follow include/bohrium/bh_ir.hpp:30-107 of the reference. Boost serialisation is not
// provided; a flat wire encoding for foreign callers is declared in include/bh_b200.h.
#pragma once

#include <cstdint>
#include <set>
#include <vector>
#include <bohrium/bh_instruction.hpp>

class BhIR {
public:
    std::vector<bh_instruction> instr_list;
    std::set<bh_base *> _syncs;
    uint64_t _nrepeats;
    // Repeat while this single BH_BOOL element is true (nullptr: no condition).
    bh_base *_repeat_condition;
    BhIR(std::vector<bh_instruction> instr_list, std::set<bh_base *> syncs, uint64_t nrepeats = 1,
         bh_base *repeat_condition = nullptr)
        : instr_list(std::move(instr_list)), _syncs(std::move(syncs)), _nrepeats(nrepeats),
          _repeat_condition(repeat_condition) {}

    const std::set<bh_base *> getSyncs() const { return _syncs; }
    uint64_t getNRepeats() const { return _nrepeats; }
    bh_base *getRepeatCondition() { return _repeat_condition; }
};

// Execution hints for a BhIR, kept beside it rather than inside it so that the BhIR keeps the
// reference's layout. A caller that executes the same, unmodified BhIR more than once registers
// them under the BhIR's address; engines look them up at every execution, and a BhIR that nobody
// registered gets the defaults, which mean "unknown" and change nothing.
//   fingerprint  a content fingerprint of the instruction list, syncs and repeat settings (0:
//                unknown): an engine may use it to recognise a repeated flush without scanning
//                the instruction list.
//   plain        the list has no sliding views and no extension-method opcodes (ids above
//                BH_MAX_OPCODE_ID), so the per-execution walks that look for them can be skipped.
// The caller clears the entry when it changes or destroys the BhIR. The table is shared by the
// whole process and safe to use from several threads.
struct BhIRHints {
    uint64_t fingerprint = 0;
    bool plain = false;
};
void bh_ir_hints_set(const BhIR *ir, const BhIRHints &hints);
BhIRHints bh_ir_hints_get(const BhIR *ir);
void bh_ir_hints_clear(const BhIR *ir);
