// Test-infrastructure shim: boost::lexical_cast<std::string> via ostringstream.
#ifndef ORACLE_SHIM_BOOST_LEXICAL_CAST_HPP
#define ORACLE_SHIM_BOOST_LEXICAL_CAST_HPP
#include <sstream>
#include <string>
namespace boost {
template <typename To, typename From> To lexical_cast(const From &v) {
    std::ostringstream os;
    os << v;
    std::istringstream is(os.str());
    To out;
    is >> out;
    return out;
}
template <> inline std::string lexical_cast<std::string>(const std::string &v) { return v; }
}
#endif
