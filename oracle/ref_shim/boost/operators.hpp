/* Stand-in for the operator-generating base classes of Boost.Operators that
   STIR's coordinate headers derive from.  The compiled file only uses the
   operators the STIR classes define themselves, so empty bases suffice. */
#ifndef ORACLE_SHIM_BOOST_OPERATORS_HPP
#define ORACLE_SHIM_BOOST_OPERATORS_HPP
namespace boost {
template <class T, class U = T> struct partially_ordered {};
template <class T, class U = T> struct equality_comparable {};
template <class T, class U = T> struct less_than_comparable {};
template <class T, class U = T> struct totally_ordered {};
}
#endif
