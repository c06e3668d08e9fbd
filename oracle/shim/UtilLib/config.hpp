// Stand-in for the CMake-generated UtilLib/config.hpp (reference build only).
#ifndef MPILIB_CONFIG_HPP_
#define MPILIB_CONFIG_HPP_
#ifndef DEBUGLEVEL
#define DEBUGLEVEL logDEBUG1
#endif
#endif
