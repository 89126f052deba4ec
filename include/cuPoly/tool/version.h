// cuPoly's include/cuPoly/tool/version.h: the library's version string.
#ifndef CUPOLYVERSION_H
#define CUPOLYVERSION_H
#include <cupoly_b200.h>

#include <string>

inline std::string GET_CUPOLY_VERSION() { return std::string("cupoly_b200 ") + cp_version(); }
#endif
