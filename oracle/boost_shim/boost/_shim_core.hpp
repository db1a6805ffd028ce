// Project-written, std-only stand-in for the small part of Boost that the
// MTL4 hot-path headers use (type traits, MPL integral constants and
// selection, enable_if, shared_ptr, tuple, unordered containers).  It exists
// only so the oracle can compile the reference headers unchanged; it is not
// part of the product library.
#ifndef MTL4_B200_BOOST_SHIM_CORE
#define MTL4_B200_BOOST_SHIM_CORE
#include <type_traits>
#include <utility>
#include <memory>
#include <tuple>
#include <complex>
#include <cstddef>
#include <cassert>
#include <climits>

namespace boost {
namespace mpl {
    template <bool B> using bool_ = std::integral_constant<bool, B>;
    typedef bool_<true>  true_;
    typedef bool_<false> false_;

    template <int N> struct int_ : std::integral_constant<int, N> {
        typedef int_ type;
        typedef int_<N + 1> next;
        typedef int_<N - 1> prior;
    };
    template <long N> struct long_ : std::integral_constant<long, N> { typedef long_ type; };
    template <typename T, T N> struct integral_c : std::integral_constant<T, N> { typedef integral_c type; };

    struct void_ { typedef void_ type; };
    struct na {};

    template <bool C, typename T1, typename T2> struct if_c { typedef T1 type; };
    template <typename T1, typename T2> struct if_c<false, T1, T2> { typedef T2 type; };
    template <typename C, typename T1, typename T2> struct if_ : if_c<bool(C::value), T1, T2> {};

    template <typename C, typename F1, typename F2>
    struct eval_if : if_<C, F1, F2>::type {};
    template <bool C, typename F1, typename F2>
    struct eval_if_c : if_c<C, F1, F2>::type {};

    template <typename T> struct identity { typedef T type; };

    template <typename... Ts> struct and_ : bool_<std::conjunction<Ts...>::value> {};
    template <typename... Ts> struct or_  : bool_<std::disjunction<Ts...>::value> {};
    template <typename T> struct not_ : bool_<!bool(T::value)> {};

    template <typename A, typename B> struct less : bool_<(A::value < B::value)> {};
    template <typename A, typename B> struct less_equal : bool_<(A::value <= B::value)> {};
    template <typename A, typename B> struct greater : bool_<(A::value > B::value)> {};
    template <typename A, typename B> struct greater_equal : bool_<(A::value >= B::value)> {};
    template <typename A, typename B> struct equal_to : bool_<(A::value == B::value)> {};
    template <typename A, typename B> struct max : if_c<(A::value < B::value), B, A> {};
    template <typename A, typename B> struct min : if_c<(B::value < A::value), B, A> {};
    template <typename A, typename B> struct plus : int_<int(A::value + B::value)> {};
    template <typename A, typename B> struct minus : int_<int(A::value - B::value)> {};

    template <typename K, typename V> struct pair { typedef K first; typedef V second; typedef pair type; };

    // Type map: a list of pair<K,V>; lookups by key with std::is_same.
    template <typename... Ps> struct map { typedef map type; };

    template <typename Map, typename K> struct at;
    template <typename K> struct at<map<>, K> { typedef void_ type; };
    template <typename P, typename... Ps, typename K>
    struct at<map<P, Ps...>, K>
      : if_c<std::is_same<typename P::first, K>::value,
             identity<typename P::second>, at<map<Ps...>, K> >::type {};

    template <typename Map, typename K> struct erase_key;
    template <typename K> struct erase_key<map<>, K> { typedef map<> type; };
    template <typename P, typename... Ps, typename K>
    struct erase_key<map<P, Ps...>, K> {
        typedef typename erase_key<map<Ps...>, K>::type rest;
        template <typename R> struct prepend;
        template <typename... Rs> struct prepend<map<Rs...> > { typedef map<P, Rs...> type; };
        typedef typename if_c<std::is_same<typename P::first, K>::value, identity<rest>, prepend<rest> >::type::type type;
    };

    template <typename Map, typename PosOrPair, typename Pair = na> struct insert;
    template <typename... Ps, typename Pos, typename P> struct insert<map<Ps...>, Pos, P> { typedef map<Ps..., P> type; };
    template <typename... Ps, typename P> struct insert<map<Ps...>, P, na> { typedef map<Ps..., P> type; };

    // Integer-indexed type sequence lookup (used with mpl::vector-like lists).
    template <typename... Ts> struct vector { typedef vector type; };
    template <typename Seq, long N> struct at_c;
    template <typename T, typename... Ts> struct at_c<vector<T, Ts...>, 0> { typedef T type; };
    template <typename T, typename... Ts, long N> struct at_c<vector<T, Ts...>, N> : at_c<vector<Ts...>, N - 1> {};
} // namespace mpl

    template <typename T> struct is_complex : std::false_type {};
    template <typename T> struct is_complex<std::complex<T> > : std::true_type {};
    template <typename T> struct is_complex<const T> : is_complex<T> {};

    using std::is_same; using std::is_const; using std::is_integral; using std::is_floating_point;
    using std::is_scalar; using std::is_unsigned; using std::is_signed; using std::is_base_of;
    using std::is_arithmetic; using std::is_pointer; using std::is_reference; using std::is_class;
    using std::is_fundamental; using std::is_convertible; using std::is_enum; using std::is_array;
    using std::remove_const; using std::remove_reference; using std::remove_pointer; using std::remove_cv;
    using std::make_signed; using std::make_unsigned; using std::add_const; using std::integral_constant;
    template <typename T> struct add_reference : std::add_lvalue_reference<T> {};
    using std::add_pointer; using std::is_void; using std::is_volatile;
    template <typename T> struct is_POD : std::bool_constant<std::is_trivial<T>::value && std::is_standard_layout<T>::value> {};
    template <typename T> struct is_pod : is_POD<T> {};
    template <typename T> struct remove_bounds : std::remove_extent<T> {};
    template <typename T> struct has_trivial_destructor : std::is_trivially_destructible<T> {};

    template <bool B, typename T = void> struct enable_if_c { typedef T type; };
    template <typename T> struct enable_if_c<false, T> {};
    template <typename C, typename T = void> struct enable_if : enable_if_c<bool(C::value), T> {};
    template <bool B, typename T = void> struct disable_if_c { typedef T type; };
    template <typename T> struct disable_if_c<true, T> {};
    template <typename C, typename T = void> struct disable_if : disable_if_c<bool(C::value), T> {};
    template <bool B, typename T> struct lazy_enable_if_c { typedef typename T::type type; };
    template <typename T> struct lazy_enable_if_c<false, T> {};
    template <typename C, typename T> struct lazy_enable_if : lazy_enable_if_c<bool(C::value), T> {};
    template <bool B, typename T> struct lazy_disable_if_c { typedef typename T::type type; };
    template <typename T> struct lazy_disable_if_c<true, T> {};
    template <typename C, typename T> struct lazy_disable_if : lazy_disable_if_c<bool(C::value), T> {};

    using std::shared_ptr;
    using std::tie; using std::get; using std::make_tuple;
    namespace tuples { using std::tuple; using std::tie; using std::get; using std::make_tuple; }
    using std::tuple;

    template <typename Target, typename Source>
    inline Target numeric_cast(Source s) { return static_cast<Target>(s); }

    class noncopyable {
      protected:
        noncopyable() {}
        ~noncopyable() {}
      private:
        noncopyable(const noncopyable&) = delete;
        noncopyable& operator=(const noncopyable&) = delete;
    };
} // namespace boost

#define BOOST_STATIC_ASSERT(...) static_assert((__VA_ARGS__), #__VA_ARGS__)
#define BOOST_STATIC_ASSERT_MSG(c, m) static_assert((c), m)
#define BOOST_ASSERT(e) assert(e)
#define BOOST_PREVENT_MACRO_SUBSTITUTION
#endif
