// Test infrastructure: compiled (not run) by tests/test_allen_shim.py against the reference's
// own headers. Allen's compile-time sequence machinery - the scheduler with its argument
// dependencies (stream/gear/include/Scheduler.cuh) and RunSequenceTuple, which calls every
// algorithm's set_arguments_size and visit (stream/gear/include/SchedulerMachinery.cuh), as
// Stream::run_sequence does (stream/sequence/src/Stream.cu:46-83) - instantiated over the
// unmodified list of configuration/sequences/Velo.h, with the VELO algorithms of
// cuda_hlt_b200/allen/VeloB200Sequence.cuh in place of the reference's.
#include <tuple>

#include "GlobalEventCut.cuh"
#include "InitEventList.cuh"
#include "VeloB200Sequence.cuh"

#define SEQUENCE_T(...) typedef std::tuple<__VA_ARGS__> configured_sequence_t;
#include "Velo.h"

#include "OutputArguments.cuh"
#include "Scheduler.cuh"
#include "SchedulerMachinery.cuh"
#include "SequenceVisitor.cuh"

using scheduler_t = Scheduler<configured_sequence_t, output_arguments_t>;

void run_velo_sequence(
  scheduler_t& scheduler,
  SequenceVisitor& visitor,
  const RuntimeOptions& runtime_options,
  const Constants& constants,
  HostBuffers& host_buffers,
  cudaStream_t& stream,
  cudaEvent_t& event)
{
  Sch::RunSequenceTuple<
    scheduler_t,
    SequenceVisitor,
    configured_sequence_t,
    std::tuple<const RuntimeOptions&, const Constants&, const HostBuffers&>,
    std::tuple<const RuntimeOptions&, const Constants&, HostBuffers&, cudaStream_t&, cudaEvent_t&>>::
    run(
      scheduler,
      visitor,
      scheduler.sequence_tuple,
      runtime_options,
      constants,
      host_buffers,
      runtime_options,
      constants,
      host_buffers,
      stream,
      event);
}
