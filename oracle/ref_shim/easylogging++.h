// TEST INFRASTRUCTURE ONLY — a stand-in for the easylogging++ interface the reference
// uses (its submodule is empty here), written for this project.  Log lines are dropped,
// except ERROR and FATAL ones, which go to stderr when STEPS_SHIM_LOG is set.
#pragma once
// The real header includes these standard headers; code that logs relies on them.
#include <algorithm>
#include <cctype>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

namespace el {
enum class Level { Global = 1, Trace, Debug, Fatal, Error, Warning, Verbose, Info, Unknown };
enum class ConfigurationType {
    Enabled, ToFile, ToStandardOutput, Format, Filename, SubsecondPrecision, MillisecondsWidth,
    PerformanceTracking, MaxLogFileSize, LogFlushThreshold, Unknown
};
enum class LoggingFlag {
    NewLineForContainer = 1, AllowVerboseIfModuleNotSpecified, LogDetailedCrashReason,
    DisableApplicationAbortOnFatalLog, ImmediateFlush, StrictLogFileSizeCheck, ColoredTerminalOutput,
    MultiLoggerSupport, DisablePerformanceTrackingCheckpointComparison, DisableVModules,
    DisableVModulesExtensions, HierarchicalLogging, CreateLoggerAutomatically, AutoSpacing,
    FixedTimeFormat, IgnoreSigInt
};
class Configurations {
  public:
    void setToDefault() {}
    void setGlobally(ConfigurationType, const std::string&) {}
    void set(Level, ConfigurationType, const std::string&) {}
    bool parseFromText(const std::string&) { return true; }
};
class Logger {
  public:
    void configure(const Configurations&) {}
};
class Loggers {
  public:
    static Logger* getLogger(const std::string&, bool = true) {
        static Logger l;
        return &l;
    }
    static void addFlag(LoggingFlag) {}
    static void removeFlag(LoggingFlag) {}
    static Logger* reconfigureLogger(const std::string& n, const Configurations&) { return getLogger(n); }
    static void reconfigureAllLoggers(const Configurations&) {}
    static void setDefaultConfigurations(const Configurations&, bool = false) {}
};
}  // namespace el

namespace steps_shim_log {
struct line {
    bool on;
    std::ostringstream os;
    explicit line(bool loud) : on(loud && std::getenv("STEPS_SHIM_LOG") != nullptr) {}
    ~line() {
        if (on) std::cerr << os.str() << std::endl;
    }
    template <class T>
    line& operator<<(const T& v) {
        if (on) os << v;
        return *this;
    }
    line& operator<<(std::ostream& (*f)(std::ostream&)) {
        if (on) os << f;
        return *this;
    }
};
constexpr bool loud(const char* lvl) {
    return lvl[0] == 'E' || lvl[0] == 'F';
}
}  // namespace steps_shim_log

#define INITIALIZE_EASYLOGGINGPP
#define CLOG(LEVEL, ...) steps_shim_log::line(steps_shim_log::loud(#LEVEL))
#define CLOG_IF(COND, LEVEL, ...) if (COND) CLOG(LEVEL)
#define CLOG_N_TIMES(N, LEVEL, ...) CLOG(LEVEL)
#define CLOG_EVERY_N(N, LEVEL, ...) CLOG(LEVEL)
