// bcc_robot_fetch.cu -- the checker pipeline instantiated for the Fetch robot.
#include "bcc.h"
#include "robot_fetch.h"
#include "bcc_pipeline.cuh"

namespace bcc {

__constant__ DevTables<FetchModel> c_tab_fetch;

template <>
__device__ __forceinline__ const DevTables<FetchModel>& tab<FetchModel>() {
    return c_tab_fetch;
}

static cudaError_t upload_fetch_tables() {
    const DevTables<FetchModel> t = host_tables<FetchModel>();
    return cudaMemcpyToSymbol(c_tab_fetch, &t, sizeof(t));
}

extern const RobotOps kFetchOps = robot_ops_of<FetchModel>(BCC_ROBOT_FETCH, upload_fetch_tables);

}  // namespace bcc
