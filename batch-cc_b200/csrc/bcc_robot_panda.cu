// bcc_robot_panda.cu -- the checker pipeline instantiated for the Panda robot.
#include "bcc.h"
#include "robot_panda.h"
#include "bcc_pipeline.cuh"

namespace bcc {

__constant__ DevTables<PandaModel> c_tab_panda;

template <>
__device__ __forceinline__ const DevTables<PandaModel>& tab<PandaModel>() {
    return c_tab_panda;
}

static cudaError_t upload_panda_tables() {
    const DevTables<PandaModel> t = host_tables<PandaModel>();
    return cudaMemcpyToSymbol(c_tab_panda, &t, sizeof(t));
}

extern const RobotOps kPandaOps = robot_ops_of<PandaModel>(BCC_ROBOT_PANDA, upload_panda_tables);

}  // namespace bcc
