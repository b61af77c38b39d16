/*
 * Minimal stand-in for easylogging++, used only to build the reference
 * (dgQuEST) from its sources for the oracle. TEST INFRASTRUCTURE ONLY.
 * LOG(WARNING|ERROR) print to stderr, LOG(FATAL) prints and aborts, lower
 * levels are dropped.
 */
#ifndef DGQ_REF_SHIM_EASYLOGGING_H
#define DGQ_REF_SHIM_EASYLOGGING_H
#include <cstdlib>
#include <iostream>
#include <sstream>

namespace el {
enum class Level { Trace, Debug, Info, Warning, Error, Fatal };
enum class LoggingFlag { ColoredTerminalOutput };
struct Loggers {
    static void addFlag(LoggingFlag) {}
    static void setLoggingLevel(Level) {}
};
}  // namespace el

namespace dgq_shim_log {
struct Line {
    int level;
    std::ostringstream os;
    explicit Line(int lv) : level(lv) {}
    ~Line() {
        if (level >= 3) std::cerr << os.str() << std::endl;
        if (level >= 5) std::abort();
    }
    template <class T>
    Line &operator<<(const T &v) {
        os << v;
        return *this;
    }
};
}  // namespace dgq_shim_log

#define DGQ_SHIM_LV_TRACE 0
#define DGQ_SHIM_LV_DEBUG 1
#define DGQ_SHIM_LV_INFO 2
#define DGQ_SHIM_LV_WARNING 3
#define DGQ_SHIM_LV_ERROR 4
#define DGQ_SHIM_LV_FATAL 5
#define LOG(lv) dgq_shim_log::Line(DGQ_SHIM_LV_##lv)
#define LOG_IF(cond, lv) if (cond) dgq_shim_log::Line(DGQ_SHIM_LV_##lv)
#define INITIALIZE_EASYLOGGINGPP
#endif
