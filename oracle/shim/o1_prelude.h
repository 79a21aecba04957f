/* Force-included into every O1 translation unit (TEST INFRASTRUCTURE).
 * Pulls in the standard headers the reference uses (it relied on macOS libc++
 * including several of them transitively), then opens the reference's private
 * members to the harness.  Standard headers are included first so the macro
 * never reaches them. */
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <iterator>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <ranges>
#include <set>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>
#define private public
