// Declaration-only header for the reference's common/intersect.cc (test infrastructure).
//
// The reference tree #includes "intersect.h" from common/intersect.cc:1 but does not ship
// it.  This header is written for this project: it only declares the SetIntersection class
// whose member definitions are in common/intersect.cc:3-981, with the signatures read off
// those definitions, so that the reference's own AVX2 set-intersection code (SI == 0) can be
// compiled unmodified into oracle/_ref/ and used as the timed CPU reference.
#pragma once
#include <immintrin.h>
#include <cstddef>
#include <cstdint>
#include "common.h"

#ifndef SI
#define SI 0
#endif

class SetIntersection {
 public:
  static size_t galloping_cnt_;
  static size_t merge_cnt_;

  static void ComputeCandidates(const vidType* larray, const vidType l_count,
                                const vidType* rarray, const vidType r_count, vidType* cn,
                                vidType& cn_count);
  static vidType get_num(const vidType* larray, const vidType l_count, const vidType* rarray,
                         const vidType r_count);

  // SI == 0 (AVX2)
  static void ComputeCNGallopingAVX2(const vidType* larray, const vidType l_count,
                                     const vidType* rarray, const vidType r_count, vidType* cn,
                                     vidType& cn_count);
  static vidType ComputeCNGallopingAVX2(const vidType* larray, const vidType l_count,
                                        const vidType* rarray, const vidType r_count);
  static void ComputeCNMergeBasedAVX2(const vidType* larray, const vidType l_count,
                                      const vidType* rarray, const vidType r_count, vidType* cn,
                                      vidType& cn_count);
  static vidType CountMergeBasedAVX2(const vidType* larray, const vidType l_count,
                                     const vidType* rarray, const vidType r_count);
  static const vidType BinarySearchForGallopingSearchAVX2(const vidType* array,
                                                          vidType offset_beg,
                                                          vidType offset_end, vidType val);
  static const vidType GallopingSearchAVX2(const vidType* array, vidType offset_beg,
                                           vidType offset_end, vidType val);
};
