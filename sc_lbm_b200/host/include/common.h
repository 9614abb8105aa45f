#ifndef COMMON_H
#define COMMON_H

// Standard headers the sc_lbm drop-in exposes to drivers (the reference's
// include/common.h pulls in the same set).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#endif
