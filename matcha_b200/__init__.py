"""matcha_b200: B200-native subtomogram-alignment hot path of Matcha.

Drop-in classes for the reference's orientation search and correlation path live in
``matcha_b200.core`` under the reference's module and class names.  All compute runs
in the CUDA library built from ``matcha_b200/csrc`` (see ``matcha_b200.build``).
"""
__version__ = "0.1.0"
