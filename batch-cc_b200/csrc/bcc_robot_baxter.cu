// bcc_robot_baxter.cu -- the checker pipeline instantiated for the Baxter robot.
#include "bcc.h"
#include "robot_baxter.h"
#include "bcc_pipeline.cuh"

namespace bcc {

__constant__ DevTables<BaxterModel> c_tab_baxter;

template <>
__device__ __forceinline__ const DevTables<BaxterModel>& tab<BaxterModel>() {
    return c_tab_baxter;
}

static cudaError_t upload_baxter_tables() {
    const DevTables<BaxterModel> t = host_tables<BaxterModel>();
    return cudaMemcpyToSymbol(c_tab_baxter, &t, sizeof(t));
}

extern const RobotOps kBaxterOps = robot_ops_of<BaxterModel>(BCC_ROBOT_BAXTER, upload_baxter_tables);

}  // namespace bcc
