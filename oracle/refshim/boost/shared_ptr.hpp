// Test infrastructure: a stand-in for boost's shared pointers, so that the reference's encoders
// compile without boost (oracle/Makefile, target refenc).  boost::shared_ptr and its casts behave
// as their std:: counterparts for every use the reference makes of them.
#pragma once
#include <memory>
#include <tuple>
#include <stdexcept>  // boost's headers bring it in; the encoders rely on that
namespace boost {
using std::shared_ptr;
using std::make_shared;
using std::static_pointer_cast;
using std::dynamic_pointer_cast;
using std::const_pointer_cast;
using std::reinterpret_pointer_cast;
}  // namespace boost
