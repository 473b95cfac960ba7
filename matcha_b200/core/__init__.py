"""Host-side mirror of ``matcha.core``: same classes, arguments and errors."""
