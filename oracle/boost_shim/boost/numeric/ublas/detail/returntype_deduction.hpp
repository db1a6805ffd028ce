// std-based stand-in for uBLAS's sizeof-based return-type deduction.  The
// result type of an arithmetic expression is located in a fixed candidate
// list (the two operand types first, then the built-in arithmetic and
// std::complex types); `test` returns a char array whose size encodes the
// position.  Only what MTL4's concept emulation reads is provided.
#ifndef MTL4_B200_SHIM_RETURNTYPE_DEDUCTION
#define MTL4_B200_SHIM_RETURNTYPE_DEDUCTION
#include <boost/_shim_core.hpp>

namespace boost { namespace numeric { namespace ublas { namespace type_deduction_detail {

template <typename T, typename... List> struct index_of;
template <typename T, typename... Rest> struct index_of<T, T, Rest...> { static const std::size_t value = 0; };
template <typename T, typename H, typename... Rest> struct index_of<T, H, Rest...>
{ static const std::size_t value = 1 + index_of<T, Rest...>::value; };

template <typename X, typename Y>
struct candidates
{
    template <template <typename...> class F>
    using apply = F<X, Y, bool, char, signed char, unsigned char, short, unsigned short, int, unsigned,
                    long, unsigned long, long long, unsigned long long, float, double, long double,
                    std::complex<float>, std::complex<double>, std::complex<long double> >;
};

template <typename... Ts> using id_vector = boost::mpl::vector<boost::mpl::identity<Ts>...>;

template <typename X, typename Y>
struct base_result_of
{
    typedef typename std::remove_cv<typename std::remove_reference<X>::type>::type x_type;
    typedef typename std::remove_cv<typename std::remove_reference<Y>::type>::type y_type;
    typedef typename candidates<x_type, y_type>::template apply<id_vector> types;
};

template <typename T, typename X, typename Y>
struct position
{
    template <typename... Ts> struct in { static const std::size_t value = index_of<T, Ts...>::value; };
    static const std::size_t value = candidates<X, Y>::template apply<in>::value;
};

template <typename X, typename Y, typename T>
char (&test(const T&))[position<typename std::remove_cv<T>::type, X, Y>::value + 1];

}}}} // namespace boost::numeric::ublas::type_deduction_detail
#endif
