// Views and instructions: shape manipulation (reshape, remove_axis, transpose), the principal
// shape of an instruction and the instruction dependency test.
// Semantics follow core/bh_view.cpp:35-192 and core/bh_instruction.cpp:34-286 of the reference.
#include <algorithm>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <bohrium/bh_instruction.hpp>

using namespace std;

uint64_t bh_base::getLabel() const { return reinterpret_cast<uint64_t>(this); }

string bh_base::str() const {
    stringstream ss;
    ss << "a" << getLabel() << "{dtype: " << bh_type_text(_type) << ", nelem: " << _nelem << "}";
    return ss.str();
}

ostream &operator<<(ostream &out, const bh_base &b) { return out << b.str(); }

bh_view::bh_view(const bh_view &view) {
    base = view.base;
    if (base == nullptr) return; // a constant operand: the remaining fields are unused
    start = view.start;
    ndim = view.ndim;
    shape = view.shape;
    stride = view.stride;
    slides = view.slides;
}

void bh_view::insert_axis(int64_t dim, int64_t size, int64_t str) {
    shape.insert(shape.begin() + dim, size);
    stride.insert(stride.begin() + dim, str);
    ++ndim;
}

void bh_view::remove_axis(int64_t dim) {
    shape.erase(shape.begin() + dim);
    stride.erase(stride.begin() + dim);
    --ndim;
}

void bh_view::transpose(int64_t axis1, int64_t axis2) {
    std::swap(shape[axis1], shape[axis2]);
    std::swap(stride[axis1], stride[axis2]);
    slides.transpose(axis1, axis2);
}

bool bh_view::isContiguous() const {
    if (isConstant()) return false;
    int64_t weight = 1;
    for (int64_t dim = ndim - 1; dim >= 0; --dim) {
        if (shape[dim] > 1 && stride[dim] != weight) return false;
        weight *= shape[dim];
    }
    return true;
}

vector<tuple<int64_t, int64_t, int64_t>> bh_view::python_notation() const {
    vector<tuple<int64_t, int64_t, int64_t>> sns; // (stride, shape, dim)
    for (int64_t i = 0; i < ndim; ++i) sns.emplace_back(stride[i], shape[i], i);
    sort(sns.begin(), sns.end(), greater<tuple<int64_t, int64_t, int64_t>>());
    vector<tuple<int64_t, int64_t, int64_t>> sne(sns.size());
    int64_t offset = start;
    for (const auto &t : sns) {
        const int64_t st = get<0>(t), sh = get<1>(t), idx = get<2>(t);
        int64_t s = st > 0 ? offset / st : 0;
        offset -= s * st;
        sne[idx] = make_tuple(s, s + sh, st);
    }
    if (offset > 0) sne.emplace_back(1, 2, offset);
    return sne;
}

string bh_view::pprint(bool py_notation) const {
    stringstream ss;
    if (isConstant()) return "CONST";
    ss << "a" << base->getLabel() << "[";
    if (py_notation) {
        const auto sne = python_notation();
        for (size_t i = 0; i < sne.size(); ++i) {
            if (i) ss << ",";
            ss << get<0>(sne[i]) << ":" << get<1>(sne[i]) << ":" << get<2>(sne[i]);
        }
    } else {
        ss << "start: " << start << ", ndim: " << ndim << ", shape: " << shape << ", stride: " << stride;
    }
    ss << "]";
    return ss.str();
}

ostream &operator<<(ostream &out, const bh_view &v) { return out << v.pprint(true); }

bool bh_view_same_shape(const bh_view *a, const bh_view *b) {
    if (a->ndim != b->ndim) return false;
    for (int64_t i = 0; i < a->ndim; ++i)
        if (a->shape[i] != b->shape[i]) return false;
    return true;
}

bool bh_view_disjoint(const bh_view *a, const bh_view *b) { return a->base != b->base; }

// --------------------------------------------------------------------------------------------
set<bh_base *> bh_instruction::get_bases() {
    set<bh_base *> ret;
    for (const bh_view &v : getViews()) ret.insert(v.base);
    return ret;
}

bool bh_instruction::isContiguous() const {
    for (const bh_view &v : getViews())
        if (!v.isContiguous()) return false;
    return true;
}

bool bh_instruction::all_same_shape() const {
    if (operand.empty()) return true;
    const bh_view &first = operand[0];
    for (size_t o = 1; o < operand.size(); ++o) {
        if (!operand[o].isConstant() && !bh_view_same_shape(&first, &operand[o])) return false;
    }
    return true;
}

bool bh_instruction::reshapable() const {
    return all_same_shape() && isContiguous() && !bh_opcode_is_sweep(opcode);
}

BhIntVec bh_instruction::shape() const {
    if (bh_opcode_is_sweep(opcode)) return operand.at(1).shape; // the swept input
    if (opcode == BH_GATHER || opcode == BH_SCATTER || opcode == BH_COND_SCATTER) return operand.at(2).shape;
    if (operand.empty()) return BhIntVec();
    return operand[0].shape;
}

int64_t bh_instruction::ndim() const { return static_cast<int64_t>(shape().size()); }

int bh_instruction::sweep_axis() const {
    if (bh_opcode_is_sweep(opcode)) return static_cast<int>(constant.get_int64());
    return BH_MAXDIM;
}

void bh_instruction::reshape(const vector<int64_t> &new_shape) {
    if (!reshapable()) throw runtime_error("Reshape: instruction not reshapable!");
    const int64_t total = accumulate(new_shape.begin(), new_shape.end(), int64_t{1}, multiplies<int64_t>());
    for (bh_view &view : getViews()) {
        if (total != view.shape.prod()) throw runtime_error("Reshape: shape mismatch!");
        view.ndim = static_cast<int64_t>(new_shape.size());
        view.shape = BhIntVec(new_shape.begin(), new_shape.end());
        view.stride.resize(new_shape.size());
        int64_t s = 1;
        for (int64_t i = view.ndim - 1; i >= 0; --i) {
            view.stride[i] = s;
            s *= view.shape[i];
        }
    }
}

void bh_instruction::remove_axis(int64_t axis) {
    if (operand.empty()) return;
    for (size_t o = 1; o < operand.size(); ++o) {
        if (!(operand[o].isConstant() || (o == 1 && opcode == BH_GATHER))) operand[o].remove_axis(axis);
    }
    const int sa = sweep_axis();
    if (sa == axis) throw runtime_error("remove_axis(): cannot remove an axis that is swept");
    if (sa > axis && sa < BH_MAXDIM) constant.set_double(sa - 1);
    if (opcode == BH_SCATTER || opcode == BH_COND_SCATTER) return; // output may have any shape
    bh_view &view = operand[0];
    if (bh_opcode_is_reduction(opcode)) {
        view.remove_axis(sa < axis ? axis - 1 : axis);
    } else {
        view.remove_axis(axis);
    }
}

void bh_instruction::transpose(int64_t axis1, int64_t axis2) {
    if (operand.empty()) return;
    for (size_t o = 1; o < operand.size(); ++o) {
        bh_view &view = operand[o];
        if (!view.isConstant() && !(o == 1 && opcode == BH_GATHER)) view.transpose(axis1, axis2);
    }
    bh_view &view = operand[0];
    const int sa = sweep_axis();
    if (sa == axis1) {
        constant.set_double(axis2);
    } else if (sa == axis2) {
        constant.set_double(axis1);
    }
    if (opcode == BH_SCATTER || opcode == BH_COND_SCATTER) return;
    if (bh_opcode_is_reduction(opcode)) {
        if (sa != axis1 && sa != axis2) {
            const int64_t t1 = sa < axis1 ? axis1 - 1 : axis1;
            const int64_t t2 = sa < axis2 ? axis2 - 1 : axis2;
            view.transpose(t1, t2);
        } else {
            // The reduced axis is one of the two: move the remaining one through a dummy axis.
            if (sa != axis1) std::swap(axis1, axis2);
            view.insert_axis(axis1, 1, 1);
            view.transpose(axis1, axis2);
            view.remove_axis(axis2);
        }
    } else {
        view.transpose(axis1, axis2);
    }
}

void bh_instruction::transpose() {
    int64_t lc = 0, rc = ndim() - 1;
    while (lc < rc) transpose(lc++, rc--);
}

bh_type bh_instruction::operand_type(int idx) const {
    const bh_view &view = operand.at(idx);
    return view.isConstant() ? constant.type : view.base->dtype();
}

string bh_instruction::pprint(bool py_notation) const {
    stringstream ss;
    if (opcode > BH_MAX_OPCODE_ID) {
        ss << "ExtMethod";
    } else {
        ss << bh_opcode_text(opcode);
    }
    for (const bh_view &v : operand) {
        ss << " ";
        if (v.isConstant()) {
            ss << constant;
        } else {
            ss << v.pprint(py_notation);
        }
    }
    return ss.str();
}

ostream &operator<<(ostream &out, const bh_instruction &instr) { return out << instr.pprint(true); }

bool bh_instr_dependency(const bh_instruction *a, const bh_instruction *b) {
    if (a->operand.empty() || b->operand.empty()) return false;
    for (const bh_view &v : a->operand)
        if (!v.isConstant() && !b->operand[0].isConstant() && !bh_view_disjoint(&b->operand[0], &v)) return true;
    for (const bh_view &v : b->operand)
        if (!v.isConstant() && !a->operand[0].isConstant() && !bh_view_disjoint(&a->operand[0], &v)) return true;
    return false;
}
