// Forced into every reference translation unit: the two Boost macros the
// reference's GPU path expands (check_CUDA.h, hoNDArray.hxx, cuNDArray.h).
#pragma once
#define BOOST_THROW_EXCEPTION(x) throw(x)
#define BOOST_CURRENT_FUNCTION __PRETTY_FUNCTION__
