// TEST STAND-IN for eWoms' ewoms/common/exceptions.hh: the one exception type the GPU drop-in
// headers throw.
#ifndef EWG_TEST_STANDIN_EXCEPTIONS_HH
#define EWG_TEST_STANDIN_EXCEPTIONS_HH

#include <stdexcept>
#include <string>

namespace Ewoms {
class NumericalIssue : public std::runtime_error
{
public:
    explicit NumericalIssue(const std::string& message) : std::runtime_error(message) {}
};
}  // namespace Ewoms

#endif
