// Test infrastructure: see log4cplus/loggingmacros.h.
#pragma once
#include "log4cplus/loggingmacros.h"
