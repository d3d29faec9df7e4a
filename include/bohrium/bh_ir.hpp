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
    // Optional content fingerprint set by a caller that executes the same, unmodified BhIR more
    // than once (0: unknown). An engine may use it to recognise a repeated flush without scanning
    // the instruction list; the caller must reset it to 0 if it changes the BhIR. (Not part of the
    // reference's BhIR; callers that never set it see no difference.)
    uint64_t _fingerprint = 0;
    // Set by a caller that knows the list has no sliding views and no extension-method opcodes
    // (ids above BH_MAX_OPCODE_ID): an engine can then skip the per-execution walks over every
    // instruction that look for them. False (unknown) by default; not part of the reference.
    bool _plain = false;

    BhIR(std::vector<bh_instruction> instr_list, std::set<bh_base *> syncs, uint64_t nrepeats = 1,
         bh_base *repeat_condition = nullptr)
        : instr_list(std::move(instr_list)), _syncs(std::move(syncs)), _nrepeats(nrepeats),
          _repeat_condition(repeat_condition) {}

    const std::set<bh_base *> getSyncs() const { return _syncs; }
    uint64_t getNRepeats() const { return _nrepeats; }
    bh_base *getRepeatCondition() { return _repeat_condition; }
};
