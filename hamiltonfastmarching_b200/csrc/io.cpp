// Key-value store with the reference IO semantics. See io.hpp.
#include "io.hpp"

#include <cstdio>
#include <iostream>
#include <sstream>

#include "../../include/hfm_b200.h"

namespace hfm {

static const char *kOrderNames[] = {"RowMajor", "ColumnMajor", "YXZ_RowMajor", "YXZ_ColumnMajor"};

const char *ordering_name(Ordering o) { return kOrderNames[static_cast<int>(o)]; }

bool ordering_from_name(const std::string &s, Ordering *o) {
    for (int i = 0; i < 4; ++i)
        if (s == kOrderNames[i]) { *o = static_cast<Ordering>(i); return true; }
    return false;
}

void Store::msg(const std::string &m) const { std::cout << m << std::flush; }
void Store::warn(const std::string &m) const {
    std::cout << "***** Warning ! *****\n" << m << "********************\n" << std::flush;
}

// ---------------------------------------------------------------- raw access (BaseIO.hxx:36-128)

bool Store::has_field(const std::string &key) const {
    if (elems_.count(key)) return true;
    visited_unset_.insert(key);
    return false;
}

bool Store::erase_field(const std::string &key) {
    unused_.erase(key);
    return elems_.erase(key) != 0;
}

const RawElement &Store::raw(const std::string &key, bool for_use) const {
    auto it = elems_.find(key);
    if (it == elems_.end()) throw Error(HFM_ERR_KEY, "BaseIO import error : field " + key + " not found.");
    if (for_use) unused_.erase(key);
    return it->second;
}

RawElement &Store::create(const std::string &key) {
    auto it = elems_.find(key);
    if (it != elems_.end()) {
        if (verbosity >= 1) warn("BaseIO: redefining field " + key + ".\n");
        it->second = RawElement();
        it->second.setter = current_setter;
    } else {
        it = elems_.emplace(key, RawElement()).first;
        it->second.setter = current_setter;
    }
    unused_.insert(key);
    return it->second;
}

std::string Store::get_string(const std::string &key) const {
    const RawElement &r = raw(key);
    if (r.count() != 0) throw Error(HFM_ERR_KEY, "BaseIO import error : field " + key + " is not a string.");
    return r.str;
}

void Store::set_string(const std::string &key, const std::string &val) { create(key).str = val; }

void Store::set_scalar(const std::string &key, double v) {
    RawElement &r = create(key);
    r.data.assign(1, v);
}

void Store::set_array(const std::string &key, const double *data, const std::vector<int64_t> &dims) {
    int64_t n = 1;
    for (int64_t d : dims) {
        if (d < 0) throw Error(HFM_ERR_VALUE, "negative extent for field " + key);
        n *= d;
    }
    RawElement &r = create(key);
    r.dims = dims;
    r.data.assign(data, data + n);
}

void Store::set_array_view(const std::string &key, const double *data, const std::vector<int64_t> &dims) {
    int64_t n = 1;
    for (int64_t d : dims) {
        if (d < 0) throw Error(HFM_ERR_VALUE, "negative extent for field " + key);
        n *= d;
    }
    if (n > 0 && !data) throw Error(HFM_ERR_ARG, "null data for field " + key);
    RawElement &r = create(key);  // a fresh element: no copied data
    r.dims = dims;
    r.ext = n > 0 ? data : nullptr;
    r.ext_n = (size_t)n;
}

std::string Store::computed_keys() const {
    std::ostringstream oss;
    oss << "[";
    for (const auto &kv : elems_)
        if (kv.second.setter == Setter::Compute)
            oss << "['" << kv.first << "','"
                << (kv.second.is_string() ? "string" : kv.second.is_scalar() ? "float" : "array") << "'],";
    oss << "]";
    return oss.str();
}

void Store::usage_report() {
    // BaseIO::UsageReport (BaseIO.hxx:64-104)
    const Setter saved = current_setter;
    current_setter = Setter::Compute;
    if (!unused_.empty()) {
        std::ostringstream ou, oc;
        for (const std::string &k : unused_) {
            auto it = elems_.find(k);
            if (it == elems_.end()) continue;
            if (it->second.setter == Setter::User) ou << k << " ";
            else oc << k << " ";
        }
        const std::string fu = ou.str(), fc = oc.str();
        if (!fu.empty()) {
            set_string("unusedFromUser", fu);
            if (verbosity >= 1) warn("Unused fields from user: " + fu + "\n");
        }
        if (!fc.empty()) {
            set_string("unusedFromCompute", fc);
            if (verbosity >= 2) msg("Unused fields from compute : " + fc + "\n");
        }
    }
    if (!defaulted_.empty()) {
        std::ostringstream o;
        for (const std::string &k : defaulted_) o << k << " ";
        set_string("defaulted", o.str());
        if (verbosity >= 2) msg("Defaulted fields : " + o.str() + "\n");
    }
    if (!visited_unset_.empty()) {
        std::ostringstream o;
        for (const std::string &k : visited_unset_) o << k << " ";
        set_string("visitedUnset", o.str());
        if (verbosity >= 3) msg("Visited but unset fields : " + o.str() + "\n");
    }
    current_setter = saved;
}

// ---------------------------------------------------------------- typed getters (IO.hxx:33-132)

static std::string fmt_double(double v) {
    std::ostringstream o;
    o << v;
    return o.str();
}

double Store::get_scalar(const std::string &key) const {
    const RawElement &r = raw(key);
    if (r.is_string()) throw Error(HFM_ERR_KEY, "IO error : key " + key + " is a string, not a numerical field.");
    if (!r.dims.empty())
        throw Error(HFM_ERR_KEY, "IO::Get error : Field " + key + " has incorrect dimensions for this object.");
    return r.ptr()[0];
}

double Store::get_scalar(const std::string &key, double def, int verb) const {
    if (has_field(key)) return get_scalar(key);
    if (verbosity >= verb) msg("Field " + key + " defaults to " + fmt_double(def) + "\n");
    visited_unset_.erase(key);
    defaulted_.insert(key);
    return def;
}

std::string Store::get_string(const std::string &key, const std::string &def, int verb) const {
    if (elems_.count(key)) return get_string(key);
    if (verbosity >= verb) msg("Field " + key + " defaults to " + def + "\n");
    visited_unset_.erase(key);
    defaulted_.insert(key);
    return def;
}

std::vector<double> Store::get_vector(const std::string &key, int ncomp, int64_t *count) const {
    const RawElement &r = raw(key);
    if (r.is_string()) throw Error(HFM_ERR_KEY, "IO error : key " + key + " is a string, not a numerical field.");
    std::vector<int64_t> dims = r.dims;
    if (ncomp > 1) {
        if (dims.empty() || dims.back() != ncomp)
            throw Error(HFM_ERR_VALUE, "BaseIO input error first dimension " +
                                           std::to_string(dims.empty() ? 0 : dims.back()) + " of field " + key +
                                           " does not match expected value " + std::to_string(ncomp) + ".");
        dims.pop_back();
    }
    if (dims.size() != 1)
        throw Error(HFM_ERR_VALUE, "IO::GetArray error : Field " + key + " has depth " + std::to_string(dims.size()) +
                                       " instead of expected 1.");
    *count = dims[0];
    return std::vector<double>(r.ptr(), r.ptr() + r.count());
}

// Element permutations of the four orderings (IO.hxx:87-110, 153-233).
static std::vector<int64_t> transpose_dims(std::vector<int64_t> d) {
    if (d.size() >= 2) std::swap(d[0], d[1]);
    return d;
}
static std::vector<int64_t> reverse_dims(std::vector<int64_t> d) {
    const size_t n = d.size();
    for (size_t i = 0; i < n / 2; ++i) std::swap(d[i], d[n - 1 - i]);
    return d;
}
static void unravel(int64_t lin, const std::vector<int64_t> &dims, std::vector<int64_t> &idx) {
    idx.resize(dims.size());
    for (int a = (int)dims.size() - 1; a >= 0; --a) { idx[a] = lin % dims[a]; lin /= dims[a]; }
}
static int64_t ravel(const std::vector<int64_t> &idx, const std::vector<int64_t> &dims) {
    int64_t r = 0;
    for (size_t a = 0; a < dims.size(); ++a) r = r * dims[a] + idx[a];
    return r;
}

// result[i] = src[ a.Convert( F(ta.Convert(i)) ) ]: a = src dims, ta = result dims.
template <typename F>
static void permute(const double *src, const std::vector<int64_t> &sdims, const std::vector<int64_t> &rdims,
                    int ncomp, double *dst, F f) {
    int64_t n = 1;
    for (int64_t d : rdims) n *= d;
    std::vector<int64_t> idx;
    for (int64_t i = 0; i < n; ++i) {
        unravel(i, rdims, idx);
        const int64_t s = ravel(f(idx), sdims);
        for (int c = 0; c < ncomp; ++c) dst[i * ncomp + c] = src[s * ncomp + c];
    }
}

std::vector<int64_t> Store::field_domain_dims(const std::string &key, int ncomp) const {
    const RawElement &r = raw(key);
    if (r.is_string()) throw Error(HFM_ERR_KEY, "IO error : key " + key + " is a string, not a numerical field.");
    std::vector<int64_t> dims = r.dims;
    if (ncomp > 1) {
        if (dims.empty() || dims.back() != ncomp)
            throw Error(HFM_ERR_VALUE, "BaseIO input error first dimension " +
                                           std::to_string(dims.empty() ? 0 : dims.back()) + " of field " + key +
                                           " does not match expected value " + std::to_string(ncomp) + ".");
        dims.pop_back();
    }
    switch (ordering_) {
        case Ordering::RowMajor: return dims;
        case Ordering::YXZ_RowMajor: return transpose_dims(dims);
        case Ordering::ColumnMajor: return reverse_dims(dims);
        case Ordering::YXZ_ColumnMajor: return transpose_dims(reverse_dims(dims));
    }
    return dims;
}

Field Store::get_field(const std::string &key, int ndim, int ncomp) const {
    const RawElement &r = raw(key);
    if (r.is_string()) throw Error(HFM_ERR_KEY, "IO error : key " + key + " is a string, not a numerical field.");
    std::vector<int64_t> sd = r.dims;
    if (ncomp > 1) {
        if (sd.empty() || sd.back() != ncomp)
            throw Error(HFM_ERR_VALUE, "BaseIO input error first dimension " +
                                           std::to_string(sd.empty() ? 0 : sd.back()) + " of field " + key +
                                           " does not match expected value " + std::to_string(ncomp) + ".");
        sd.pop_back();
    }
    Field f;
    f.ncomp = ncomp;
    if (sd.empty()) {  // DataSource_Value
        f.data.assign(r.ptr(), r.ptr() + ncomp);
        return f;
    }
    if ((int)sd.size() != ndim)
        throw Error(HFM_ERR_VALUE, "IO::GetArray error : Field " + key + " has depth " + std::to_string(sd.size()) +
                                       " instead of expected " + std::to_string(ndim) + ".");
    int64_t n = 1;
    for (int64_t d : sd) n *= d;
    if (ordering_ != Ordering::RowMajor) f.data.resize(n * ncomp);
    switch (ordering_) {
        case Ordering::RowMajor:
            f.dims = sd;
            f.data.clear();
            f.view = r.ptr();
            break;
        case Ordering::YXZ_RowMajor:
            f.dims = transpose_dims(sd);
            permute(r.ptr(), sd, f.dims, ncomp, f.data.data(),
                    [](const std::vector<int64_t> &i) { return transpose_dims(i); });
            break;
        case Ordering::ColumnMajor:
            f.dims = reverse_dims(sd);
            permute(r.ptr(), sd, f.dims, ncomp, f.data.data(),
                    [](const std::vector<int64_t> &i) { return reverse_dims(i); });
            break;
        case Ordering::YXZ_ColumnMajor:
            f.dims = transpose_dims(reverse_dims(sd));
            permute(r.ptr(), sd, f.dims, ncomp, f.data.data(),
                    [](const std::vector<int64_t> &i) { return reverse_dims(transpose_dims(i)); });
            break;
    }
    return f;
}

void Store::set_field(const std::string &key, const std::vector<int64_t> &dims, int ncomp, const double *data) {
    std::vector<int64_t> od;
    std::vector<double> out;
    int64_t n = 1;
    for (int64_t d : dims) n *= d;
    out.resize(n * ncomp);
    switch (ordering_) {
        case Ordering::RowMajor:
            od = dims;
            std::copy(data, data + n * ncomp, out.begin());
            break;
        case Ordering::YXZ_RowMajor:
            od = transpose_dims(dims);
            permute(data, dims, od, ncomp, out.data(), [](const std::vector<int64_t> &i) { return transpose_dims(i); });
            break;
        case Ordering::ColumnMajor:
            od = reverse_dims(dims);
            permute(data, dims, od, ncomp, out.data(), [](const std::vector<int64_t> &i) { return reverse_dims(i); });
            break;
        case Ordering::YXZ_ColumnMajor:
            od = reverse_dims(transpose_dims(dims));
            permute(data, dims, od, ncomp, out.data(),
                    [](const std::vector<int64_t> &i) { return transpose_dims(reverse_dims(i)); });
            break;
    }
    if (ncomp > 1) od.push_back(ncomp);
    set_array(key, out.data(), od);
}

double *Store::create_field(const std::string &key, const std::vector<int64_t> &dims, int ncomp) {
    if (ordering_ != Ordering::RowMajor) return nullptr;
    int64_t n = ncomp;
    for (int64_t d : dims) n *= d;
    RawElement &r = create(key);
    r.dims = dims;
    if (ncomp > 1) r.dims.push_back(ncomp);
    r.data.resize(n);
    return r.data.data();
}

void Store::set_vector(const std::string &key, int64_t count, int ncomp, const double *data) {
    std::vector<int64_t> d{count};
    if (ncomp > 1) d.push_back(ncomp);
    set_array(key, data, d);
}

}  // namespace hfm
