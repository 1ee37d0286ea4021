// Same include path as the reference header; the API lives in scopi_gpu.hpp.
#pragma once
#include "../scopi_gpu.hpp"
