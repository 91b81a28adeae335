// cudf/aggregation.hpp -- aggregation kinds and factories with the reference's
// names and enum values (cpp/include/cudf/aggregation.hpp:86-124, 199, 261-411).
#pragma once

#include <memory>
#include <vector>

#include "types.hpp"

namespace cudf {

class aggregation {
 public:
  enum Kind {
    SUM, PRODUCT, MIN, MAX, COUNT_VALID, COUNT_ALL, ANY, ALL, SUM_OF_SQUARES, MEAN, M2, VARIANCE, STD,
    MEDIAN, QUANTILE, ARGMAX, ARGMIN, NUNIQUE, NTH_ELEMENT, ROW_NUMBER, EWMA, RANK, COLLECT_LIST,
    COLLECT_SET, LEAD, LAG, PTX, CUDA, MERGE_LISTS, MERGE_SETS, MERGE_M2, COVARIANCE, CORRELATION,
    TDIGEST, MERGE_TDIGEST, HISTOGRAM, MERGE_HISTOGRAM
  };
  aggregation() = delete;
  explicit aggregation(Kind a) : kind{a} {}
  virtual ~aggregation() = default;
  Kind kind;
  size_type ddof{1};                                    // VARIANCE / STD; n of NTH_ELEMENT
  null_policy null_handling{null_policy::EXCLUDE};      // NUNIQUE / NTH_ELEMENT
  interpolation interp{interpolation::LINEAR};          // QUANTILE
  std::vector<double> quantiles;                        // QUANTILE
};

class groupby_aggregation : public virtual aggregation {
 public:
  explicit groupby_aggregation(Kind k) : aggregation(k) {}
};

namespace detail {
template <typename Base>
std::unique_ptr<Base> make_agg(aggregation::Kind k, size_type ddof = 1)
{
  auto p  = std::make_unique<groupby_aggregation>(k);
  p->ddof = ddof;
  return std::unique_ptr<Base>(p.release());
}
}  // namespace detail

template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_sum_aggregation() { return detail::make_agg<Base>(aggregation::SUM); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_product_aggregation() { return detail::make_agg<Base>(aggregation::PRODUCT); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_min_aggregation() { return detail::make_agg<Base>(aggregation::MIN); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_max_aggregation() { return detail::make_agg<Base>(aggregation::MAX); }
// COUNT_VALID for EXCLUDE, COUNT_ALL for INCLUDE (cpp/src/aggregation/aggregation.cpp:494-499)
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_count_aggregation(null_policy null_handling = null_policy::EXCLUDE)
{
  return detail::make_agg<Base>(null_handling == null_policy::EXCLUDE ? aggregation::COUNT_VALID
                                                                      : aggregation::COUNT_ALL);
}
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_sum_of_squares_aggregation() { return detail::make_agg<Base>(aggregation::SUM_OF_SQUARES); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_mean_aggregation() { return detail::make_agg<Base>(aggregation::MEAN); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_variance_aggregation(size_type ddof = 1) { return detail::make_agg<Base>(aggregation::VARIANCE, ddof); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_std_aggregation(size_type ddof = 1) { return detail::make_agg<Base>(aggregation::STD, ddof); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_argmax_aggregation() { return detail::make_agg<Base>(aggregation::ARGMAX); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_argmin_aggregation() { return detail::make_agg<Base>(aggregation::ARGMIN); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_m2_aggregation() { return detail::make_agg<Base>(aggregation::M2); }
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_median_aggregation() { return detail::make_agg<Base>(aggregation::MEDIAN); }
// aggregation.hpp:364: num_groups * q.size() result rows, group by group
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_quantile_aggregation(std::vector<double> const& q, interpolation i = interpolation::LINEAR)
{
  auto p       = detail::make_agg<Base>(aggregation::QUANTILE);
  p->quantiles = q;
  p->interp    = i;
  return p;
}
// aggregation.hpp:397
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_nunique_aggregation(null_policy null_handling = null_policy::EXCLUDE)
{
  auto p           = detail::make_agg<Base>(aggregation::NUNIQUE);
  p->null_handling = null_handling;
  return p;
}
// aggregation.hpp:410-411
template <typename Base = groupby_aggregation>
std::unique_ptr<Base> make_nth_element_aggregation(size_type n, null_policy null_handling = null_policy::INCLUDE)
{
  auto p           = detail::make_agg<Base>(aggregation::NTH_ELEMENT, n);
  p->null_handling = null_handling;
  return p;
}

}  // namespace cudf
