// TEST STAND-IN for eWoms' ewoms/common/propertysystem.hh: just enough of the property and
// parameter system for the GPU drop-in headers (GpuEcfvLinearizer, GpuBiCGStabBackend) to compile
// in a test program without eWoms. A type tag is a struct whose member types are the properties
// and whose nested Params struct has one static function per runtime parameter.
#ifndef EWG_TEST_STANDIN_PROPERTYSYSTEM_HH
#define EWG_TEST_STANDIN_PROPERTYSYSTEM_HH

#define GET_PROP_TYPE(TypeTag, PropTagName) typename TypeTag::PropTagName
#define EWOMS_GET_PARAM(TypeTag, ParamType, ParamName) (static_cast<ParamType>(TypeTag::Params::ParamName()))
#define EWOMS_REGISTER_PARAM(TypeTag, ParamType, ParamName, Description) ((void)0)
#define BEGIN_PROPERTIES
#define END_PROPERTIES
#define NEW_PROP_TAG(PTagName)

#endif
