// Test infrastructure: a stand-in for boost::function.
#pragma once
#include <functional>
namespace boost {
using std::function;
}  // namespace boost
