// UtilLib::Log (libs/UtilLib/include/Log.hpp): a process-wide log stream and
// the LOG(level) macro; messages at or below the reporting level go to the
// stream set by Log::setStream, one line each.
#ifndef LBIBCELL_DROPIN_UTILLIB_LOG_HPP
#define LBIBCELL_DROPIN_UTILLIB_LOG_HPP

#include <memory>
#include <ostream>
#include <sstream>
#include <string>

namespace UtilLib {

enum LogLevel { logERROR, logWARNING, logINFO, logDEBUG, logDEBUG1, logDEBUG2, logDEBUG3, logDEBUG4 };

class Log {
 public:
    Log() {}
    ~Log();  // writes the buffered line
    std::ostringstream& writeReport(LogLevel level = logINFO);

    static std::shared_ptr<std::ostream> getStream();
    static void setStream(std::shared_ptr<std::ostream> pStream);
    static LogLevel getReportingLevel();
    static void setReportingLevel(LogLevel level);
    static void writeOutput(const std::string& msg);

 private:
    Log(const Log&);
    Log& operator=(const Log&);
    std::ostringstream buffer_;
};

}  // namespace UtilLib

#define LOG(level)                                                                        \
    if (level > UtilLib::Log::getReportingLevel() || !UtilLib::Log::getStream()) ;          \
    else UtilLib::Log().writeReport(level)

#endif
