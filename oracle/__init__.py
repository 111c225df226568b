"""CPU oracle of the SCB sweep path (test infrastructure only; see trt_oracle.cpp)."""
