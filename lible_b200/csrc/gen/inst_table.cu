// Generated by gen_instances.py: lookup of class kernels.
#include "../eri_launch.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd64_00[1];
    extern const int u_fwd64_00[1];
    extern const LaunchFn k_fwd64_01[2];
    extern const int u_fwd64_01[2];
    extern const LaunchFn k_fwd64_02[3];
    extern const int u_fwd64_02[3];
    extern const LaunchFn k_fwd64_03[4];
    extern const int u_fwd64_03[4];
    extern const LaunchFn k_fwd64_04[5];
    extern const int u_fwd64_04[5];
    extern const LaunchFn k_fwd64_05[6];
    extern const int u_fwd64_05[6];
    extern const LaunchFn k_fwd64_06[7];
    extern const int u_fwd64_06[7];
    extern const LaunchFn k_fwd64_07[8];
    extern const int u_fwd64_07[8];
    extern const LaunchFn k_fwd64_08[9];
    extern const int u_fwd64_08[9];
    extern const LaunchFn k_fwd64_09[10];
    extern const int u_fwd64_09[10];
    extern const LaunchFn k_fwd64_10[11];
    extern const int u_fwd64_10[11];
    extern const LaunchFn k_fwd64_11[12];
    extern const int u_fwd64_11[12];
    static const int *const u_fwd64[12] = {u_fwd64_00, u_fwd64_01, u_fwd64_02, u_fwd64_03, u_fwd64_04, u_fwd64_05, u_fwd64_06, u_fwd64_07, u_fwd64_08, u_fwd64_09, u_fwd64_10, u_fwd64_11};
    static const LaunchFn *const k_fwd64[12] = {k_fwd64_00, k_fwd64_01, k_fwd64_02, k_fwd64_03, k_fwd64_04, k_fwd64_05, k_fwd64_06, k_fwd64_07, k_fwd64_08, k_fwd64_09, k_fwd64_10, k_fwd64_11};
    extern const LaunchFn k_fwd32_00[1];
    extern const int u_fwd32_00[1];
    extern const LaunchFn k_fwd32_01[2];
    extern const int u_fwd32_01[2];
    extern const LaunchFn k_fwd32_02[3];
    extern const int u_fwd32_02[3];
    extern const LaunchFn k_fwd32_03[4];
    extern const int u_fwd32_03[4];
    extern const LaunchFn k_fwd32_04[5];
    extern const int u_fwd32_04[5];
    extern const LaunchFn k_fwd32_05[6];
    extern const int u_fwd32_05[6];
    extern const LaunchFn k_fwd32_06[7];
    extern const int u_fwd32_06[7];
    extern const LaunchFn k_fwd32_07[8];
    extern const int u_fwd32_07[8];
    extern const LaunchFn k_fwd32_08[9];
    extern const int u_fwd32_08[9];
    extern const LaunchFn k_fwd32_09[10];
    extern const int u_fwd32_09[10];
    static const int *const u_fwd32[10] = {u_fwd32_00, u_fwd32_01, u_fwd32_02, u_fwd32_03, u_fwd32_04, u_fwd32_05, u_fwd32_06, u_fwd32_07, u_fwd32_08, u_fwd32_09};
    static const LaunchFn *const k_fwd32[10] = {k_fwd32_00, k_fwd32_01, k_fwd32_02, k_fwd32_03, k_fwd32_04, k_fwd32_05, k_fwd32_06, k_fwd32_07, k_fwd32_08, k_fwd32_09};
    extern const LaunchFn k_d1_00[1];
    extern const LaunchFn k_d1_01[2];
    extern const LaunchFn k_d1_02[3];
    extern const LaunchFn k_d1_03[4];
    extern const LaunchFn k_d1_04[5];
    extern const LaunchFn k_d1_05[6];
    extern const LaunchFn k_d1_06[7];
    extern const LaunchFn k_d1_07[8];
    extern const LaunchFn k_d1_08[9];
    extern const LaunchFn k_d1_09[10];
    extern const LaunchFn k_d1_10[11];
    extern const LaunchFn k_d1_11[12];
    static const LaunchFn *const k_d1[12] = {k_d1_00, k_d1_01, k_d1_02, k_d1_03, k_d1_04, k_d1_05, k_d1_06, k_d1_07, k_d1_08, k_d1_09, k_d1_10, k_d1_11};
    LaunchFn lookupFwd64(int bt, int kt)
    {
        if (bt < 0 || bt >= 12 || kt < 0 || kt > bt)
            return nullptr;
        return k_fwd64[bt][kt];
    }
    LaunchFn lookupFwd32(int bt, int kt)
    {
        if (bt < 0 || bt >= 10 || kt < 0 || kt > bt)
            return nullptr;
        return k_fwd32[bt][kt];
    }
    LaunchFn lookupD1(int bt, int kt)
    {
        if (bt < 0 || bt >= 12 || kt < 0 || kt > bt)
            return nullptr;
        return k_d1[bt][kt];
    }
    int unitFwd(int bt, int kt, bool fp32)
    {
        if (bt < 0 || kt < 0 || kt > bt || bt >= (fp32 ? 10 : 12))
            return 0;
        return fp32 ? u_fwd32[bt][kt] : u_fwd64[bt][kt];
    }
}
