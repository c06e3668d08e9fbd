// UtilLib::Exception and lbm_fail for applications and plugins written
// against LBIBCell's API (libs/UtilLib/include/Exception.hpp): the same names
// and meaning, backed by lbibcell_b200's device runtime.
#ifndef LBIBCELL_DROPIN_UTILLIB_EXCEPTION_HPP
#define LBIBCELL_DROPIN_UTILLIB_EXCEPTION_HPP

#include <stdexcept>
#include <string>

namespace UtilLib {

// The library's exception: a message, and where it was raised.
class Exception : public std::exception {
 public:
    explicit Exception(const std::string& message) : message_(message) {}
    Exception(const std::string& message, const char* file, int line)
        : message_(message + " (" + file + ":" + std::to_string(line) + ")") {}
    virtual ~Exception() throw() {}
    virtual const char* what() const throw() { return message_.c_str(); }

 private:
    std::string message_;
};

}  // namespace UtilLib

#define lbm_fail(ERROR_MESSAGE) throw(UtilLib::Exception(ERROR_MESSAGE, __FILE__, __LINE__))

#endif
