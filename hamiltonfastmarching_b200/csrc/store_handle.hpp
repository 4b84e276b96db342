// The object behind the opaque hfm_io handle of the C ABI: a key-value store plus the message of
// its last failure.
#pragma once

#include <string>

#include "io.hpp"

struct hfm_io {
    hfm::Store store;
    std::string last_error;
    explicit hfm_io(hfm::Ordering o) : store(o) {}
};
