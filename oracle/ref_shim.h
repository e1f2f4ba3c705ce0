/* Force-included ahead of every reference translation unit when the
 * reference library (JonnyWideFoot/pd.arcus src/mmlib) is compiled as the
 * test oracle.  The reference's exception header uses the include guard
 * __EXCEPTION_H, which collides with libstdc++'s <bits/exception.h>; the
 * standard headers are therefore pulled in first and the guard released.
 * Nothing in the reference sources is modified. */
#include <exception>
#include <typeinfo>
#include <new>
#include <stdexcept>
#include <climits>
#include <cstring>
#include <cstdlib>
#include <cstdio>
#include <cfloat>
#include <algorithm>
#include <string>
#include <vector>
#include <iostream>
#include <fstream>
#include <sstream>
#include <valarray>
#undef __EXCEPTION_H
