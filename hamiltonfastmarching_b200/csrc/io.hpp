// Key-value store with the reference IO semantics (host side of the C ABI).
//
// Follows JMM_CPPLibs/JMM_CPPLibs/Output/BaseIO.h:16-43 / BaseIO.hxx:8-160 (raw elements, setter
// tags, the unused/defaulted/visitedUnset bookkeeping and UsageReport) and IO.hxx:33-170 (typed
// getters with defaults, the four array orderings). Internally every domain array is RowMajor
// with axes in (x, y, z|theta) order and the component axis last.
#pragma once

#include <sys/mman.h>

#include <cstdint>
#include <cstdlib>
#include <map>
#include <new>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace hfm {

// Error carrying an hfm_b200.h status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Allocator of the store's numerical arrays: blocks of 4 MiB and more are mapped directly and
// advised for transparent huge pages, so copying a large field in or out costs few page faults.
template <typename T>
struct BigAlloc {
    using value_type = T;
    static constexpr size_t kThreshold = size_t(4) << 20;
    BigAlloc() = default;
    template <typename U> BigAlloc(const BigAlloc<U> &) {}
    T *allocate(size_t n) {
        const size_t bytes = n * sizeof(T);
        if (bytes >= kThreshold) {
            void *p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
            if (p == MAP_FAILED) throw std::bad_alloc();
            madvise(p, bytes, MADV_HUGEPAGE);
            return static_cast<T *>(p);
        }
        void *p = std::malloc(bytes ? bytes : 1);
        if (!p) throw std::bad_alloc();
        return static_cast<T *>(p);
    }
    void deallocate(T *p, size_t n) {
        const size_t bytes = n * sizeof(T);
        if (bytes >= kThreshold) munmap(p, bytes);
        else std::free(p);
    }
    // resize() leaves new elements uninitialised (an output field is written in full by the solver,
    // so zero-filling hundreds of MB first would only cost page faults and bandwidth)
    template <typename U> void construct(U *p) { ::new ((void *)p) U; }
    template <typename U, typename... A> void construct(U *p, A &&...a) { ::new ((void *)p) U(std::forward<A>(a)...); }
    template <typename U> bool operator==(const BigAlloc<U> &) const { return true; }
    template <typename U> bool operator!=(const BigAlloc<U> &) const { return false; }
};
using DoubleArray = std::vector<double, BigAlloc<double>>;

enum class Setter { User, Compute, Unknown };
enum class Ordering { RowMajor = 0, ColumnMajor = 1, YXZ_RowMajor = 2, YXZ_ColumnMajor = 3 };

struct RawElement {
    std::string str;
    std::vector<int64_t> dims;
    DoubleArray data;
    // an array referenced in the caller's memory instead of `data` (set_array_view)
    const double *ext = nullptr;
    size_t ext_n = 0;
    Setter setter = Setter::Unknown;
    const double *ptr() const { return ext ? ext : data.data(); }
    size_t count() const { return ext ? ext_n : data.size(); }
    bool is_string() const { return count() == 0 && dims.empty(); }
    bool is_scalar() const { return count() != 0 && dims.empty(); }
};

// A domain field read from the store: RowMajor over `dims` (x, y, z order), `ncomp` components
// per point (component fastest). `dims` is empty for a constant field given as a single element.
// `view` points into the store when no reordering is needed (RowMajor); it stays valid until the
// field is modified or erased.
struct Field {
    std::vector<int64_t> dims;
    int ncomp = 1;
    std::vector<double> data;
    const double *view = nullptr;
    bool constant() const { return dims.empty(); }
    const double *ptr() const { return view ? view : data.data(); }
    size_t size() const {
        size_t n = (size_t)ncomp;
        for (int64_t d : dims) n *= (size_t)d;
        return n;
    }
};

class Store {
public:
    explicit Store(Ordering def) : default_ordering_(def), ordering_(def) {}

    Setter current_setter = Setter::User;
    int verbosity = 1;

    // --- raw access (BaseIO) ---
    bool has_field(const std::string &key) const;
    bool erase_field(const std::string &key);
    std::string get_string(const std::string &key) const;
    void set_string(const std::string &key, const std::string &val);
    void set_scalar(const std::string &key, double v);
    void set_array(const std::string &key, const double *data, const std::vector<int64_t> &dims);
    // Like set_array, without copying: the store reads `data` in place until the key is replaced
    // or erased (the caller keeps it alive and unmodified meanwhile).
    void set_array_view(const std::string &key, const double *data, const std::vector<int64_t> &dims);
    const RawElement &raw(const std::string &key, bool for_use = true) const;
    std::string computed_keys() const;
    void usage_report();

    // --- typed getters (IO_) ---
    double get_scalar(const std::string &key) const;
    double get_scalar(const std::string &key, double def, int verb = 1) const;
    std::string get_string(const std::string &key, const std::string &def, int verb = 1) const;
    // Vector of points / scalars: raw dims (n) or (n, ncomp); ordering does not apply to vectors.
    std::vector<double> get_vector(const std::string &key, int ncomp, int64_t *count) const;
    // Domain field: depth must be `ndim` (or 0 for a constant element); component axis last.
    Field get_field(const std::string &key, int ndim, int ncomp) const;
    std::vector<int64_t> field_domain_dims(const std::string &key, int ncomp) const;
    // Output of a RowMajor domain array (x, y, z order) with `ncomp` trailing components.
    void set_field(const std::string &key, const std::vector<int64_t> &dims, int ncomp,
                   const double *data);
    void set_vector(const std::string &key, int64_t count, int ncomp, const double *data);
    // A computed RowMajor domain array to be filled in place by the caller; nullptr when the
    // ordering requires a permutation (then use set_field).
    double *create_field(const std::string &key, const std::vector<int64_t> &dims, int ncomp);

    void set_ordering(Ordering o) { ordering_ = o; }
    Ordering ordering() const { return ordering_; }
    Ordering default_ordering() const { return default_ordering_; }

    void msg(const std::string &m) const;
    void warn(const std::string &m) const;

private:
    RawElement &create(const std::string &key);
    std::map<std::string, RawElement> elems_;
    mutable std::set<std::string> unused_, defaulted_, visited_unset_;
    Ordering default_ordering_, ordering_;
};

const char *ordering_name(Ordering o);
bool ordering_from_name(const std::string &s, Ordering *o);

}  // namespace hfm
