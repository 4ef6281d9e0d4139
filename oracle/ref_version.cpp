// Test infrastructure for oracle/_ref/libgail.so: the reference's build_version.cpp needs a
// header its CMake generates, so the version string is given here as the reference stamps
// a build made outside its own git repository (cmake/BuildVersion.cmake: the plain release
// number, "1.1.0").
namespace gail {
const char* buildVersion() { return "1.1.0"; }
}  // namespace gail
