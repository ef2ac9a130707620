// Project-wide includes of the standalone plugin build (the reference's
// src/header.hpp plays this role inside the reference tree).
#ifndef MASS_GPU_COMPAT_HEADER_HPP_
#define MASS_GPU_COMPAT_HEADER_HPP_

#include <array>
#include <cmath>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include <boost/program_options.hpp>

constexpr unsigned width = 70;

#endif
