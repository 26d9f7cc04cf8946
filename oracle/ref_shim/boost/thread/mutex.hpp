// boost::mutex (cudaDeviceManager's per-device cuBLAS lock) as std::mutex.
#pragma once
#include <mutex>
namespace boost {
using std::mutex;
}
