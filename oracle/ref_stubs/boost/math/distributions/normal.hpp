/* Stand-in for the one Boost.Math facility the reference uses (erf_inv). */
#ifndef OA_REF_BOOST_NORMAL_HPP
#define OA_REF_BOOST_NORMAL_HPP
#include <boost/math/special_functions/erf.hpp>
#endif
