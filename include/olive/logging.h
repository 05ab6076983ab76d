/*
 * olive_b200 source-compatible header layer: LOG(level) stream logging to
 * stderr with the reference's levels and names (logging.h:43-101).  The
 * reporting level defaults to DEBUG as in the reference and can be lowered
 * with Logging::ReportingLevel() = WARNING.  Not thread-safe.
 */
#ifndef OLIVE_LOGGING_H
#define OLIVE_LOGGING_H

#include <sstream>
#include <string>

#include "common.h"

enum LogLevel { ERROR = 0, WARNING, INFO, DEBUG, DEBUG1, DEBUG2, DEBUG3 };

class Logging {
    std::ostringstream os_;
    LogLevel level_ = INFO;

public:
    ~Logging() {
        if (level_ <= ReportingLevel()) {
            os_ << '\n';
            fputs(os_.str().c_str(), stderr);
            fflush(stderr);
        }
    }
    std::ostringstream &Get(LogLevel lv = INFO) {
        static const char *names[] = {"ERROR", "WARNING", "INFO", "DEBUG",
                                      "DEBUG1", "DEBUG2", "DEBUG3"};
        level_ = lv;
        os_ << ((lv >= ERROR && lv <= DEBUG3) ? names[lv] : "UNKNOWN") << ": ";
        return os_;
    }
    static LogLevel &ReportingLevel() {
        static LogLevel lv = DEBUG;
        return lv;
    }
};

#define LOG(level) Logging().Get(level)

#endif  // OLIVE_LOGGING_H
