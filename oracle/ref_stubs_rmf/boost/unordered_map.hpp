/* Stand-in: boost::unordered_map as std::unordered_map with boost::hash (see disjoint_sets.hpp). */
#pragma once
#include <unordered_map>
#include <boost/functional/hash.hpp>
namespace boost {
template <class K, class V> using unordered_map = std::unordered_map<K, V, boost::hash<K>>;
}
