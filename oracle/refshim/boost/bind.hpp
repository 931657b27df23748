// Test infrastructure: a stand-in for boost::bind and its global placeholders.
#pragma once
#include <functional>
namespace boost {
using std::bind;
}  // namespace boost
using namespace std::placeholders;
