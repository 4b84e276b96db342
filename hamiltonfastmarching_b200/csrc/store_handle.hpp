// The object behind the opaque hfm_io handle of the C ABI: a key-value store plus the message of
// its last failure.
#pragma once

#include <memory>
#include <string>

#include "io.hpp"

struct hfm_io {
    hfm::Store store;
    std::string last_error;
    std::shared_ptr<void> retained;  // device state of the last solve run with retainState = 1
    explicit hfm_io(hfm::Ordering o) : store(o) {}
};
