"""Oracle bindings (TEST INFRASTRUCTURE ONLY): the C restatement (``liboracle.so``) and, when it
was built here, the reference's own CPU engine (``_ref/libcelv2ref.so``). Only the tests, the
smoke check and the benchmark's CPU-baseline leg import this package."""
from .binding import Oracle, Reference, reference_available, records_equal, first_difference

__all__ = ["Oracle", "Reference", "reference_available", "records_equal", "first_difference"]
