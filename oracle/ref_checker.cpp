// ORACLE — test infrastructure only. Runs the reference's own VELO track checker
// (TrackCheckerVelo, checker/tracking/src/TrackChecker.cpp:349-405 with the categories of
// checker/tracking/src/CategoriesTrackChecker.cpp and the association of
// checker/tracking/include/MCAssociator.h:166-182), compiled from the reference tree without
// ROOT, on tracks and MC truth handed in as plain arrays, and returns its counters, so that
// tests can compare them with this library's velo_check_tracks.
//
// The steps around the checker are those of its callers: one MCEvent per MC_info blob
// (checker/tracking/src/MCEvent.cpp:16-148, as CheckerInvoker::read_mc_folder builds them),
// tracks as trackChecker::Tracks with the LHCb ids of each consolidated track in order (as
// prepareVeloTracks does, checker/tracking/src/PrepareTracks.cpp:14-41), then, per event,
// an MCAssociator over the event's VELO MC particles and one call of the checker
// (CheckerInvoker::check, checker/tracking/include/CheckerInvoker.h:46-64).
#include <cstdint>
#include <cstring>
#include <vector>

#include "MCAssociator.h"
#include "MCEvent.h"
#include "TrackChecker.h"

namespace {

// Reads the protected counters of the checker and of its efficiency reports.
struct CheckerProbe : TrackCheckerVelo {
  size_t n_categories() const { return m_categories.size(); }
  const TrackEffReport& report(size_t i) const { return m_categories[i]; }
  size_t tracks() const { return m_ntracks; }
  size_t ghosts() const { return m_nghosts; }
  float ghost_per_event() const { return m_ghostperevent; }
  // The reports print their results when destroyed; a report without accepted particles
  // prints nothing, so the counters are cleared once they have been read.
  void silence()
  {
    for (auto& r : m_categories) r.m_naccept = 0;
  }
};

}  // namespace

extern "C" {

// Runs TrackCheckerVelo over n_events events. mc_blob / mc_offsets: MC_info/tracks blobs
// and their u64 byte offsets; event_track_offsets[n_events + 1], track_hit_offsets[T + 1],
// hit_ids[H]: the consolidated tracks (Consolidated::Tracks offsets and LHCb ids).
// Writes, for up to max_categories categories, the name (64 bytes each, NUL-terminated) and
// counts[3 * i ..] = reconstructible, found, clones; totals = {tracks, ghosts};
// *ghost_per_event = the checker's per-event ghost average. Returns the number of categories.
int ref_check_velo_tracks(const void* mc_blob, const uint64_t* mc_offsets, uint32_t n_events,
                          const uint32_t* event_track_offsets, const uint32_t* track_hit_offsets,
                          const uint32_t* hit_ids, uint32_t max_categories, char* names, uint64_t* counts,
                          uint64_t* totals, float* ghost_per_event)
{
  const char* base = static_cast<const char*>(mc_blob);
  CheckerProbe checker;
  for (uint32_t e = 0; e < n_events; ++e) {
    const std::vector<char> blob(base + mc_offsets[e], base + mc_offsets[e + 1]);
    const MCEvent mc_event(blob, false);
    trackChecker::Tracks tracks;
    for (uint32_t t = event_track_offsets[e]; t < event_track_offsets[e + 1]; ++t) {
      trackChecker::Track track;
      track.p = 0.f;
      for (uint32_t h = track_hit_offsets[t]; h < track_hit_offsets[t + 1]; ++h) track.addId(hit_ids[h]);
      tracks.push_back(track);
    }
    const auto& mcps = mc_event.mc_particles<TrackCheckerVelo>();
    MCAssociator mcassoc {mcps};
    checker(tracks, mcassoc, mcps);
  }
  const size_t n = checker.n_categories();
  for (size_t i = 0; i < n && i < max_categories; ++i) {
    const auto& r = checker.report(i);
    std::strncpy(names + 64 * i, r.m_name.c_str(), 63);
    names[64 * i + 63] = 0;
    counts[3 * i] = r.m_naccept;
    counts[3 * i + 1] = r.m_nfound;
    counts[3 * i + 2] = r.m_nclones;
  }
  totals[0] = checker.tracks();
  totals[1] = checker.ghosts();
  *ghost_per_event = checker.ghost_per_event();
  checker.silence();
  return static_cast<int>(n);
}

}  // extern "C"
