/* Work-item id storage for the OpenCL builtin shim (oracle only). */
namespace oclshim {
thread_local int g_gid[2];
thread_local int g_lid[2];
thread_local int g_lsize[2] = {1, 1};
thread_local int g_grp[2];
}  // namespace oclshim
