/*
 * Minimal stand-in for <boost/tuple/tuple.hpp>, used only to compile the
 * reference's own hot-path sources into the CPU oracle (oracle/_ref).
 * Test infrastructure, not product code.  boost::tuple<T...> is modelled as
 * a std::tuple with the member accessor get<N>() that boost provides.
 */
#ifndef ORACLE_SHIM_BOOST_TUPLE_HPP
#define ORACLE_SHIM_BOOST_TUPLE_HPP
#include <tuple>

namespace boost {
template <typename... T>
class tuple : public std::tuple<T...> {
 public:
  using std::tuple<T...>::tuple;
  tuple() : std::tuple<T...>() {}
  template <int N>
  typename std::tuple_element<N, std::tuple<T...>>::type& get() { return std::get<N>(*this); }
  template <int N>
  const typename std::tuple_element<N, std::tuple<T...>>::type& get() const { return std::get<N>(*this); }
};
template <int N, typename... T>
typename std::tuple_element<N, std::tuple<T...>>::type& get(tuple<T...>& t) { return std::get<N>(t); }
template <int N, typename... T>
const typename std::tuple_element<N, std::tuple<T...>>::type& get(const tuple<T...>& t) { return std::get<N>(t); }
namespace tuples { using boost::get; }
}  // namespace boost
#endif
