/* Test infrastructure (oracle reference build): VarsTools is used only by
 * code off the operator path; declarations for it to parse. */
#ifndef SHIM_VARSTOOLS_HPP_
#define SHIM_VARSTOOLS_HPP_
namespace VarsTools
{
template <class mapping_function_t, class var_t>
void define_enum_mapping(mapping_function_t mapping_function, int ivar,
                         var_t &var)
{
    mapping_function(ivar, var);
}
template <class vars_t, class value_t> void assign(vars_t &, const value_t &)
{
}
} // namespace VarsTools
#endif
