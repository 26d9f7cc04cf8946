// Header-only stand-in for the Boost smart pointers the reference's GPU path
// uses (boost::shared_ptr / make_shared / pointer casts): the C++17 standard
// library equivalents under the boost namespace.  Test infrastructure only.
#pragma once
#include <memory>
namespace boost {
using std::const_pointer_cast;
using std::dynamic_pointer_cast;
using std::enable_shared_from_this;
using std::make_shared;
using std::shared_ptr;
using std::static_pointer_cast;
using std::weak_ptr;
}  // namespace boost
