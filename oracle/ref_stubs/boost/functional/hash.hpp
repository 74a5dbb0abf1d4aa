/* Stand-in: boost::hash with the one use the reference makes of it (hashing std::pair). */
#pragma once
#include <cstddef>
#include <functional>
#include <utility>
namespace boost {
template <typename T> struct hash;
template <typename A, typename B> struct hash<std::pair<A, B>> {
    std::size_t operator()(const std::pair<A, B>& p) const {
        return std::hash<A>()(p.first) * 31u + std::hash<B>()(p.second);
    }
};
}
