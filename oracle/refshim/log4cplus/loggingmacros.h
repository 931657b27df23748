// Test infrastructure: a stand-in for log4cplus that discards every message, so that the
// reference's encoders compile without the library.  Only the names the encoders use exist.
#pragma once
#include <string>
namespace log4cplus {
class Logger {
public:
    static Logger getRoot() { return Logger(); }
    static Logger getInstance(const std::string &) { return Logger(); }
};
namespace helpers {}
}  // namespace log4cplus
#define LOG4CPLUS_TEXT(x) x
#define LOG4CPLUS_FATAL(l, m) do { } while (0)
#define LOG4CPLUS_ERROR(l, m) do { } while (0)
#define LOG4CPLUS_WARN(l, m) do { } while (0)
#define LOG4CPLUS_INFO(l, m) do { } while (0)
#define LOG4CPLUS_DEBUG(l, m) do { } while (0)
#define LOG4CPLUS_TRACE(l, m) do { } while (0)
#define LOG4CPLUS_INFO_FMT(l, ...) do { } while (0)
#define LOG4CPLUS_DEBUG_FMT(l, ...) do { } while (0)
#define LOG4CPLUS_TRACE_FMT(l, ...) do { } while (0)
#define LOG4CPLUS_WARN_FMT(l, ...) do { } while (0)
#define LOG4CPLUS_ERROR_FMT(l, ...) do { } while (0)
