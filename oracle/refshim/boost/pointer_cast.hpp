// Test infrastructure: see boost/shared_ptr.hpp.
#pragma once
#include "boost/shared_ptr.hpp"
