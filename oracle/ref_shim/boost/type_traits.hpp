// The reference includes boost/type_traits.hpp but uses only std traits.
#pragma once
#include <type_traits>
