// Test infrastructure: a stand-in for boost::scoped_ptr (a non-copyable owning pointer).
#pragma once
#include <memory>
namespace boost {
template <class T>
using scoped_ptr = std::unique_ptr<T>;
}  // namespace boost
