// Test infrastructure: a stand-in for boost::is_same.
#pragma once
#include <type_traits>
namespace boost {
using std::is_same;
}  // namespace boost
