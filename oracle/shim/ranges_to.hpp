// Test-infrastructure shim, force-included into the oracle build of the
// reference's CPU grower: the C++23 `std::ranges::to<C>()` pipe adaptor,
// which g++ 13's libstdc++ lacks. Covers the one form that code uses
// (a view piped into `to<std::vector<T>>()`).
#pragma once

#include <ranges>
#include <version>

#if !defined(__cpp_lib_ranges_to_container)
namespace std::ranges
{
namespace shim_detail
{
template <typename C> struct to_adaptor
{
};

template <typename R, typename C> C operator|(R &&r, to_adaptor<C>)
{
    C out;
    for (auto &&v : r)
    {
        out.push_back(static_cast<typename C::value_type>(v));
    }
    return out;
}
} // namespace shim_detail

template <typename C> shim_detail::to_adaptor<C> to()
{
    return {};
}
} // namespace std::ranges
#endif
