/* Stand-in for the reference's build of src/recursiveMedianFiltering.cpp: the union-find and
 * property-map names its colour-guided fill is written with.  Only the plain fill
 * (recursiveMedianFilterAux) of that file is run from this build; the colour-guided function
 * merely has to compile. */
#pragma once
#include <utility>
namespace boost {
template <class Map> struct associative_property_map {
    Map* m;
    explicit associative_property_map(Map& x) : m(&x) {}
};
template <class Map> associative_property_map<Map> make_assoc_property_map(Map& m)
{
    return associative_property_map<Map>(m);
}
template <class RankMap, class ParentMap> class disjoint_sets {
    RankMap rank_;
    ParentMap parent_;

  public:
    disjoint_sets(RankMap r, ParentMap p) : rank_(r), parent_(p) {}
    template <class E> void make_set(E x) { (*parent_.m)[x] = x; (*rank_.m)[x] = 0; }
    template <class E> E find_set(E x)
    {
        while (!((*parent_.m)[x] == x)) x = (*parent_.m)[x];
        return x;
    }
    template <class E> void union_set(E a, E b)
    {
        a = find_set(a);
        b = find_set(b);
        if (!(a == b)) (*parent_.m)[b] = a;
    }
};
}  // namespace boost
