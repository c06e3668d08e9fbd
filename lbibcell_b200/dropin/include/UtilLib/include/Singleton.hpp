// UtilLib::Singleton (libs/UtilLib/include/Singleton.hpp): one instance of T
// per process, created on first use.
#ifndef LBIBCELL_DROPIN_UTILLIB_SINGLETON_HPP
#define LBIBCELL_DROPIN_UTILLIB_SINGLETON_HPP

namespace UtilLib {

template <class T>
class Singleton {
 public:
    static T& instance() {
        static T object;
        return object;
    }

 private:
    Singleton();
};

}  // namespace UtilLib

#endif
