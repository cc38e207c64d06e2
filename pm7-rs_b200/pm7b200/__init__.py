"""B200 PM7/NDDO SCF engine: Python host API over the C ABI of include/pm7_b200.h."""
