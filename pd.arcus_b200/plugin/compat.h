/* Pre-included when the component compiles against the PD headers with a
 * current g++: PD's exception.h guards itself with __EXCEPTION_H, the same
 * guard libstdc++'s <bits/exception.h> uses, so the standard headers PD
 * relies on are included first and the guard is released again. */
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
#include <map>
#include <iostream>
#include <fstream>
#include <sstream>
#include <valarray>
#undef __EXCEPTION_H
